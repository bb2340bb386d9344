// Stage kernels of convective flux 3 (fluxFunction = 3).
#define CCFD_FLUX_ID 3
#include "stage_flux.inc"
