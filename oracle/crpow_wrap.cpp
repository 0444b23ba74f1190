// crpow_wrap.cpp -- TEST INFRASTRUCTURE: pow() for a build of the reference
// linked with -Wl,--wrap=pow (oracle/Makefile, _ref/libcrpropa_crpow.so).
// Every pow call of the reference's own sources then goes to the correctly
// rounded pow of the engine's FP64 form (crpropa3_b200/csrc/crmath.cuh), so
// that adaptive step controllers (PropagationCK.cpp:111, PropagationBP.cpp:117)
// can be compared with the device bit for bit; everything else is the
// reference's own arithmetic.  Inputs outside cr_pow's range go to the C
// library's pow (__real_pow).
#include <cmath>

extern "C" double __real_pow(double, double);
#define pow __real_pow
#include "crmath.cuh"
#undef pow

extern "C" double __wrap_pow(double x, double y) { return crp::cr_pow(x, y); }
