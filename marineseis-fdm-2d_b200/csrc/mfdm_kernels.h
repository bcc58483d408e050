// Host-side launchers of the time-step kernels (internal to the library).
#pragma once
#include <cuda_runtime.h>

#include "mfdm_device.cuh"

namespace mfdm {

// Sets the dynamic shared-memory limit of every stage kernel on the current device.
cudaError_t configure_device();
// Launches RK stage `stage` (0..3) with operator direction `dir` (0 = F, 1 = B).
// Stage 0 reads `in` == U^n; stages 1-2 read `in` and U^n (`un`); stage 3 writes U.
// `maps` holds the TMA descriptors of this stage's input, U^n, accumulator and coefficients.
cudaError_t launch_stage(const Coef& C, const Fields& in, const Fields& out, const Fields& un,
                         const Fields& acc, const StageMaps& maps, int stage, int dir,
                         cudaStream_t st);
// Interface filter, receiver sampling and step-counter advance.
cudaError_t launch_finish(const Coef& C, const Fields& U, cudaStream_t st);
// Replaces each of rows x nx floats (row pitch P) by its reciprocal, computed in
// FP64 and rounded once.
cudaError_t launch_reciprocal(float* a, int rows, int nx, int P, cudaStream_t st);
// Sets the device step counter to `it`.
cudaError_t launch_set_step(const Coef& C, int it, cudaStream_t st);
// Dynamic shared memory of one stage block.
size_t stage_smem_bytes();
// The stage build a launch uses: C.variant (2 or 3 resident ring blocks per SM,
// 4 the tile build), or the 3-block ring build when 0.
int stage_blocks_per_sm(const Coef& C);
// Default rows per segment block when C.seg is unset: 24 from 6 M cells per
// launch (fewer halo rows re-read), 8 below (more blocks than SMs on smaller
// grids); the autotuner's picks at 4096x2048, 2048x1024 and 1200x800.
inline int default_seg_rows(const Coef& C) {
  const long long cells = (long long)C.nx * (C.nzf + C.nzs) * (C.nshots > 0 ? C.nshots : 1);
  return cells >= 6000000LL ? 24 : 8;
}
// Rows per segment block of a stage launch (C.seg, or the default when unset).
int stage_seg_rows(const Coef& C);
// Block counts of one stage launch (per shot) with `seg` rows per segment:
// column tiles, fluid tiles, solid tiles, interface blocks.
void stage_grid(int nx, int nzf, int nzs, int seg, int* ntx, int* nbf, int* nbs, int* nbi);
// Uploads the 5x5 source weights and the 7-point interface filter weights.
cudaError_t upload_constants(const float* srcw25, const float* w7);

// Library-internal host helpers (mfdm_host.cu): record a failure for
// mfdm_last_error() and return `code`; encode a TMA map of a [nf][rows][P] block
// (rows_outer: boxes land as [row][field][col], the stencil-ring layout; with
// nshots > 0 a fourth dimension, the shot, of stride shot_bytes).
int set_error(int code, const char* msg);
// Ricker value at `time` in the reference's host float arithmetic: the one
// source of every Ricker table the library uploads.
float ricker_ref(float fpeak, float time);
// CFS-PML factors (d/beta, alpha + d/beta, 1/beta, 0) of cell i of an axis of n
// cells, computed in FP64 on the host: the one source of every PML table.
float4 pml_cell(float fpeak, float beta0, int npd, int npow, float vp_max, float rc,
                float thickness, int i, int n, bool lo, bool hi);
int encode_block_map(CUtensorMap* map, const float* base, int P, int rows, int nf, int box_x,
                     bool rows_outer, int nshots = 0, size_t shot_bytes = 0);

}  // namespace mfdm
