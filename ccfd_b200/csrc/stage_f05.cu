// FP64 stage kernels of convective flux 5 (fluxFunction = 5).
#define CCFD_FLUX_ID 5
#define CCFD_FLUX_FP32 0
#include "stage_flux.inc"
