// crpow.cpp -- TEST INFRASTRUCTURE: the correctly rounded pow of the
// engine's FP64 form (crpropa3_b200/csrc/crmath.cuh), exported for the oracle
// build that isolates pow's last-place differences (crp_oracle.c, ORACLE_POW).
#include "crmath.cuh"

extern "C" double oracle_cr_pow(double x, double y) { return crp::cr_pow(x, y); }
