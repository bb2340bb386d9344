// Mixed-precision stage kernels of convective flux 6 (fluxFunction = 6).
#define CCFD_FLUX_ID 6
#define CCFD_FLUX_FP32 1
#include "stage_flux.inc"
