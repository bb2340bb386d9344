// FP64 stage kernels of convective flux 3 (fluxFunction = 3).
#define CCFD_FLUX_ID 3
#define CCFD_FLUX_FP32 0
#include "stage_flux.inc"
