// FP64 stage kernels of convective flux 4 (fluxFunction = 4).
#define CCFD_FLUX_ID 4
#define CCFD_FLUX_FP32 0
#include "stage_flux.inc"
