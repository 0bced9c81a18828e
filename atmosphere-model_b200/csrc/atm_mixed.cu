// Mixed-precision form of the dynamical core: the horizontal sweeps run in
// FP32 (fields and PPM arithmetic), while the column pressure sums, pkap,
// the hydrostatic geopotential feeding the pressure-gradient force, the
// vertical remap and the global mass sum stay in FP64.
#define ATM_FORM_T float
#define ATM_OPS_NAME ops_mixed
#include "atm_launch.cuh"
