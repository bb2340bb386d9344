// Mixed-precision stage kernels of convective flux 8 (fluxFunction = 8).
#define CCFD_FLUX_ID 8
#define CCFD_FLUX_FP32 1
#include "stage_flux.inc"
