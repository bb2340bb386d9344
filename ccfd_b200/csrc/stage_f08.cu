// FP64 stage kernels of convective flux 8 (fluxFunction = 8).
#define CCFD_FLUX_ID 8
#define CCFD_FLUX_FP32 0
#include "stage_flux.inc"
