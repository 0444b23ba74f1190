"""B200-native charged-particle stepping for CRPropa3 chains.

`crpropa3_b200.engine` is the handle on the C-ABI engine (include/crp_gpu.h,
built into crpropa3_b200/lib/libcrp_b200.so for sm_100a).
"""
__version__ = "0.1.0"
