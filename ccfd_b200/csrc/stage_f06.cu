// Stage kernels of convective flux 6 (fluxFunction = 6).
#define CCFD_FLUX_ID 6
#include "stage_flux.inc"
