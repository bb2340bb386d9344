// Mixed-precision stage kernels of convective flux 3 (fluxFunction = 3).
#define CCFD_FLUX_ID 3
#define CCFD_FLUX_FP32 1
#include "stage_flux.inc"
