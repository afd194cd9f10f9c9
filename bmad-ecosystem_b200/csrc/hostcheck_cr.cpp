// hostcheck_cr.cpp -- TEST-ONLY: the host check build (hostcheck.cpp) with the correctly rounded
// transcendentals of crmath.cuh in the maps and in the element invariants (BG_CR_MATH, set on the
// command line for both translation units), i.e. the device's arithmetic on the CPU. With the
// same correctly rounded functions installed in the oracle (oracle_set_libm) the two agree bit
// for bit, which the CPU tests check before the GPU is compared with the oracle in that mode.
#define bmadgpu_hostcheck_track bmadgpu_hostcheck_cr_track
#define bmadgpu_hostcheck_last_error bmadgpu_hostcheck_cr_last_error
#include "hostcheck.cpp"
