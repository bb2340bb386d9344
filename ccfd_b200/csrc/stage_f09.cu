// FP64 stage kernels of convective flux 9 (fluxFunction = 9).
#define CCFD_FLUX_ID 9
#define CCFD_FLUX_FP32 0
#include "stage_flux.inc"
