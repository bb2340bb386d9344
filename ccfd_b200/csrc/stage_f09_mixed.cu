// Mixed-precision stage kernels of convective flux 9 (fluxFunction = 9).
#define CCFD_FLUX_ID 9
#define CCFD_FLUX_FP32 1
#include "stage_flux.inc"
