// Mixed-precision stage kernels of convective flux 2 (fluxFunction = 2).
#define CCFD_FLUX_ID 2
#define CCFD_FLUX_FP32 1
#include "stage_flux.inc"
