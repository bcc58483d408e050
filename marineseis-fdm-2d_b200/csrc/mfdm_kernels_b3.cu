// The stage kernels built for three resident blocks per SM: 4 stencil and 2
// point-wise ring slots (about 74 KB of shared memory per block) and a
// 72-register budget. Large grids stream faster this way (more bytes in flight
// per SM), small grids slower; the launchers pick per model, and the tile
// autotuner times both (mfdm_kernels.cu holds the source).
#define MFDM_VNS v3
#define MFDM_VARIANT_TU 1
#define MFDM_STENCIL_SLOTS 4
#define MFDM_PW_SLOTS 2
#define MFDM_MIN_BLOCKS 3
#include "mfdm_kernels.cu"
