// Stage kernels of convective flux 11 (fluxFunction = 11).
#define CCFD_FLUX_ID 11
#include "stage_flux.inc"
