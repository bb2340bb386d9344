// FP64 stage kernels of convective flux 10 (fluxFunction = 10).
#define CCFD_FLUX_ID 10
#define CCFD_FLUX_FP32 0
#include "stage_flux.inc"
