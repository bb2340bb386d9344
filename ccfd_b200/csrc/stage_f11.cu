// FP64 stage kernels of convective flux 11 (fluxFunction = 11).
#define CCFD_FLUX_ID 11
#define CCFD_FLUX_FP32 0
#include "stage_flux.inc"
