// Mixed-precision stage kernels of convective flux 11 (fluxFunction = 11).
#define CCFD_FLUX_ID 11
#define CCFD_FLUX_FP32 1
#include "stage_flux.inc"
