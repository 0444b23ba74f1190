"""argtypes / restype of every entry point declared in include/crp_gpu.h."""
from __future__ import annotations

import ctypes as C

from . import _abi

_u64, _i32, _u32, _d = C.c_uint64, C.c_int32, C.c_uint32, C.c_double
_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_plan_p = C.c_void_p

# name -> (restype, argtypes); the list is the C-ABI's exported surface.
SIGNATURES = {
    "crp_abi_version": (_u32, []),
    "crp_last_error": (_i32, [C.c_char_p, C.c_size_t]),
    "crp_device_count": (_i32, [_i32p]),
    "crp_plan_create": (_i32, [C.POINTER(_abi.PlanDesc), C.POINTER(_plan_p)]),
    "crp_plan_destroy": (_i32, [_plan_p]),
    "crp_run": (_i32, [_plan_p, C.POINTER(_abi.Candidates), _u64, C.POINTER(_abi.RunOpts),
                       C.POINTER(_abi.RunStats)]),
    "crp_run_device": (_i32, [_plan_p, C.POINTER(_abi.Candidates), _u64,
                              C.POINTER(_abi.RunOpts), C.POINTER(_abi.RunStats)]),
    "crp_field_eval": (_i32, [_plan_p, _u64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "crp_autotune": (_i32, [_plan_p, C.POINTER(_abi.Candidates), _u64, _u64, _u64, C.c_void_p,
                            C.POINTER(_abi.AutotuneResult)]),
    "crp_particle_charge": (_i32, [_i32, _dp]),
    "crp_bp_adjoint_workspace": (_i32, [C.POINTER(_abi.AdjointDesc), _u64, C.POINTER(C.c_size_t)]),
    "crp_bp_forward_loss": (_i32, [C.POINTER(_abi.AdjointDesc), C.POINTER(_abi.AdjointIO), C.c_void_p]),
    "crp_bp_adjoint": (_i32, [C.POINTER(_abi.AdjointDesc), C.POINTER(_abi.AdjointIO), C.c_void_p,
                              C.c_size_t, C.c_void_p]),
    "crp_bp_adjoint_forward": (_i32, [C.POINTER(_abi.AdjointDesc), C.POINTER(_abi.AdjointIO),
                                      C.c_void_p, C.c_size_t, C.c_void_p]),
    "crp_bp_adjoint_backward": (_i32, [C.POINTER(_abi.AdjointDesc), C.POINTER(_abi.AdjointIO),
                                       C.c_void_p, C.c_size_t, C.c_void_p]),
    "crp_random_draws": (_i32, [_u32, _i32, _u64, _d, _d, _d, _dp]),
    "crp_jf12_defaults": (_i32, [_i32, C.POINTER(_abi.JF12Desc)]),
    "crp_jf12_solenoidal": (_i32, [_d, _d, C.POINTER(_abi.JF12Desc)]),
    "crp_uf23_defaults": (_i32, [_i32, C.POINTER(_abi.UF23Desc)]),
    "crp_pt11_defaults": (_i32, [C.POINTER(_abi.PT11Desc)]),
    "crp_pt11_use": (_i32, [C.POINTER(_abi.PT11Desc), _i32, _i32]),
    "crp_tf17_defaults": (_i32, [_i32, _i32, C.POINTER(_abi.TF17Desc)]),
    "crp_kst24_defaults": (_i32, [C.POINTER(_abi.KST24Desc)]),
    "crp_cmz_defaults": (_i32, [C.POINTER(_abi.CMZDesc)]),
    "crp_single_mode_field": (_i32, [_d, _d, _d, C.POINTER(_d), C.POINTER(_d), C.POINTER(_d), _i32, _i32, _i32,
                                     C.POINTER(_abi.SingleModeDesc)]),
    "crp_turbulence_draws": (_i32, [_u32, _i32, _u64, _dp]),
    "crp_turbulence_modes": (_i32, [C.POINTER(_abi.TurbulenceDesc), C.POINTER(C.c_uint64)]),
    "crp_turbulence_grid": (_i32, [C.POINTER(_abi.TurbulenceDesc), C.c_void_p, C.c_void_p]),
    "crp_plane_wave_modes": (_i32, [_d, _d, _d, _d, _d, _d, _i32, _i32, _dp, _dp, _dp, _dp, _dp]),
    "crp_source_sample": (_i32, [C.c_void_p, _u32, _u64, _i32p, _dp, _dp]),
    "crp_source_sample_device": (_i32, [C.c_void_p, _u64, _u64, _u64, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p]),
    "crp_text_output_write": (_i32, [C.c_char_p, _i32, _i32, C.c_void_p, _u64, C.c_void_p]),
    "crp_run_device_noalloc": (_i32, [C.POINTER(_abi.NoAllocGridBpDesc), C.POINTER(_abi.Candidates),
                                      _u64, C.c_void_p, C.POINTER(_abi.RunStats)]),
}

# entry points added by later parts of the library, declared when present
OPTIONAL = {}


def declare(lib):
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    for name, (res, args) in OPTIONAL.items():
        if hasattr(lib, name):
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
