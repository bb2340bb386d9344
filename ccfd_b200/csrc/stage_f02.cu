// FP64 stage kernels of convective flux 2 (fluxFunction = 2).
#define CCFD_FLUX_ID 2
#define CCFD_FLUX_FP32 0
#include "stage_flux.inc"
