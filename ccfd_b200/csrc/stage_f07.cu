// FP64 stage kernels of convective flux 7 (fluxFunction = 7).
#define CCFD_FLUX_ID 7
#define CCFD_FLUX_FP32 0
#include "stage_flux.inc"
