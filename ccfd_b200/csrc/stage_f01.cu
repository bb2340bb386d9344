// FP64 stage kernels of convective flux 1 (fluxFunction = 1).
#define CCFD_FLUX_ID 1
#define CCFD_FLUX_FP32 0
#include "stage_flux.inc"
