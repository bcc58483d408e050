// Solid only with a free surface on top (the reference's PmlFs::SolidOnly,
// include/pml_fs_kernels.cuh:8-307, src/pml_fs_kernels.cu:5-381) or with
// CFS-PML on all four sides (Cpml::SolidOnly, include/cpml_kernels.cuh:8-233,
// src/cpml_kernels.cu:5-361): device data and launchers (library-internal).
#pragma once
#include <cuda_runtime.h>

namespace mfdm {
namespace solid {

// Coefficients and tables of one solid-only model. All [nz][P] arrays are
// row-major with pitch P; the free surface is row 3.
struct SCoef {
  int nx, nz, P, Ps, npd;
  const float* __restrict__ C11;
  const float* __restrict__ C13;
  const float* __restrict__ C33;
  const float* __restrict__ C55;
  const float* __restrict__ rcp_rho;  // 1/rho: FP64 reciprocal rounded once
  const float* __restrict__ J;
  const float* __restrict__ xix;
  const float* __restrict__ xiz;
  const float* __restrict__ zex;
  const float* __restrict__ zez;
  const float* __restrict__ alm;    // [6][P]: al1_xx, al1_zz, al1_xz, al2_xx, al2_zz, al2_xz (row 3)
  const float4* __restrict__ pmlx;  // per column: d/beta, alpha + d/beta, 1/beta
  const float4* __restrict__ pmlz;  // per row (bottom band; with cpml also the top band)
  const float* __restrict__ src_amp;  // Ricker value per (step, stage): [steps][4]
  int src_steps;
  int srcx, srcz;                   // source cell (srcx < 0: none)
  float rk_c[4];                    // dt/2, dt/2, dt, dt/6
  float rk_w[3];                    // dt/6, dt/3, dt/3
  int gap, rec_cap;
  float* rec;                       // [rec_cap][nx]: solid vz on row rec_row
  int rec_row;                      // 3 (free surface) or 30 (cpml), src/main.cu:303-311
  int cpml;                         // 1: CFS-PML on all four sides, no free surface
  int* step;                        // device step counter
  unsigned* done;                   // block arrival counter of the finish kernel
  int* status;                      // sticky non-finite flag
};

// One RK set: the five fields [nz][P], the xi-ADE strips [nz][Ps] (Vx, Vz, Ex,
// Ez; slot s of column 3+s or nx-3-npd+s-npd) and the zeta-ADE band [npd][P]
// (rows nz-3-npd..nz-4; with cpml [2 npd][P], the top band's rows 3..npd+2
// after the bottom band's).
struct SFields {
  float *vx, *vz, *sx, *sz, *sxz;
  float* x[4];
  float* z[4];
};

// RK stage `stage` (0..3) with operator direction `dir` (0 F, 1 B): reads `in`
// (and U^n = `un`, the accumulator `acc`), writes `out` and the accumulator.
cudaError_t launch_stage(const SCoef& C, const SFields& in, const SFields& out, const SFields& un,
                         const SFields& acc, int stage, int dir, cudaStream_t st);
// Records solid vz on row rec_row when the step index is a multiple of gap, flags
// non-finite values and advances the device step counter.
cudaError_t launch_finish(const SCoef& C, const SFields& U, cudaStream_t st);
// Sets the device step counter.
cudaError_t launch_set_step(const SCoef& C, int it, cudaStream_t st);

}  // namespace solid
}  // namespace mfdm
