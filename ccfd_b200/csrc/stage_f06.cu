// FP64 stage kernels of convective flux 6 (fluxFunction = 6).
#define CCFD_FLUX_ID 6
#define CCFD_FLUX_FP32 0
#include "stage_flux.inc"
