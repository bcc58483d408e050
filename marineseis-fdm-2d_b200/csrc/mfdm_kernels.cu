// sm_100a kernels of the fluid-solid RK4 time step.
//
// One launch per RK stage does the whole stage: the stage right-hand side of
// every fluid and solid cell (the four reference RHS kernels), the mirrored
// ghost fluxes (built on the fly from the stage input instead of a separate
// build_ghost_flux launch), the source, the interface coupling and the RK4
// bookkeeping (the 48 matrix_add / matrix_self_add launches and the 48 reset
// copies of the reference become one fused read-modify-write). A fifth launch
// per step filters the interface rows, samples the receivers and advances the
// device step counter. Reference: src/pml_fs_kernels.cu:533-868.
//
// Block roles inside one stage launch (blockIdx.x ranges):
//   [0, nbf)            fluid tiles: kTX columns x kTZ rows of fluid rows 3..nz_f-2
//   [nbf, nbf+nbs)      solid tiles: kTX columns x kTZ rows of solid rows 1..nz_s-4
//   [nbf+nbs, ...)      interface strip: one thread per column, fluid row nz_f-1
//                       and solid row 0 together, so the normal/tangential
//                       coupling happens in registers.
// Tiles stage the stencil fields of the stage input in shared memory with a
// halo of 3 rows and 4 columns (float4-aligned), so every stencil tap is a
// shared-memory read; point-wise fields (coefficients, U^n, accumulator, ADE
// strips) stream straight from HBM, coalesced along x.
#include "mfdm_device.cuh"
#include "mfdm_kernels.h"

namespace mfdm {

constexpr int kTX = 64;                 // tile width (columns)
constexpr int kTZ = 32;                 // tile height (rows)
constexpr int kThreads = 256;           // threads per block (64 x 4)
constexpr int kHX = 4, kHZ = 3;         // tile halo
constexpr int kTW = kTX + 2 * kHX;      // 72 floats per staged row
constexpr int kTH = kTZ + 2 * kHZ;      // 38 staged rows
constexpr int kRowsPerThread = kTZ / (kThreads / kTX);

struct TileAcc {
  const float* t;  // staged fields, [nf][kTH][kTW]
  int r, c;        // cell position inside the tile
  __device__ __forceinline__ float at(int f, int dz, int dx) const {
    return t[(f * kTH + r + dz) * kTW + c + dx];
  }
};
struct FluidTile : TileAcc {
  __device__ __forceinline__ float fvx(int dz, int dx) const { return at(0, dz, dx); }
  __device__ __forceinline__ float fvz(int dz, int dx) const { return at(1, dz, dx); }
  __device__ __forceinline__ float fp(int dz, int dx) const { return at(2, dz, dx); }
};
struct SolidTile : TileAcc {
  __device__ __forceinline__ float svx(int dz, int dx) const { return at(0, dz, dx); }
  __device__ __forceinline__ float svz(int dz, int dx) const { return at(1, dz, dx); }
  __device__ __forceinline__ float ssx(int dz, int dx) const { return at(2, dz, dx); }
  __device__ __forceinline__ float ssz(int dz, int dx) const { return at(3, dz, dx); }
  __device__ __forceinline__ float ssxz(int dz, int dx) const { return at(4, dz, dx); }
};
// Direct reads of the stage input (interface strip).
struct FluidGlobal {
  const float *vx, *vz, *p;
  size_t base;
  int P;
  __device__ __forceinline__ float fvx(int dz, int dx) const { return __ldg(vx + base + (ptrdiff_t)dz * P + dx); }
  __device__ __forceinline__ float fvz(int dz, int dx) const { return __ldg(vz + base + (ptrdiff_t)dz * P + dx); }
  __device__ __forceinline__ float fp(int dz, int dx) const { return __ldg(p + base + (ptrdiff_t)dz * P + dx); }
};
struct SolidGlobal {
  const float *vx, *vz, *sx, *sz, *sxz;
  size_t base;
  int P;
  __device__ __forceinline__ float svx(int dz, int dx) const { return __ldg(vx + base + (ptrdiff_t)dz * P + dx); }
  __device__ __forceinline__ float svz(int dz, int dx) const { return __ldg(vz + base + (ptrdiff_t)dz * P + dx); }
  __device__ __forceinline__ float ssx(int dz, int dx) const { return __ldg(sx + base + (ptrdiff_t)dz * P + dx); }
  __device__ __forceinline__ float ssz(int dz, int dx) const { return __ldg(sz + base + (ptrdiff_t)dz * P + dx); }
  __device__ __forceinline__ float ssxz(int dz, int dx) const { return __ldg(sxz + base + (ptrdiff_t)dz * P + dx); }
};

// Stages nf fields of rows [z0-3, z0+kTZ+3) x columns [x0-4, x0+kTX+4) into
// shared memory with float4 loads; cells outside the array read as zero.
template <int NF>
__device__ __forceinline__ void stage_tile(float* tile, const float* const (&src)[NF], int rows,
                                           int P, int x0, int z0) {
  constexpr int kQ = kTW / 4;
  for (int f = 0; f < NF; ++f) {
    const float* s = src[f];
    for (int q = threadIdx.x; q < kTH * kQ; q += kThreads) {
      const int r = q / kQ, c4 = q - r * kQ;
      const int z = z0 - kHZ + r, x = x0 - kHX + 4 * c4;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (z >= 0 && z < rows && x >= 0 && x < P)
        v = __ldg(reinterpret_cast<const float4*>(s + (size_t)z * P + x));
      *reinterpret_cast<float4*>(tile + (f * kTH + r) * kTW + 4 * c4) = v;
    }
  }
}

template <int DIR, int KIND>
__device__ __forceinline__ void fluid_tile(const Coef& C, const Fields& in, const Fields& out,
                                           const Fields& un, const Fields& acc, int s, int it,
                                           int tile, int ntx, float* sm) {
  const int nx = C.nx, P = C.P, nzf = C.nzf;
  const int x0 = (tile % ntx) * kTX, z0 = 3 + (tile / ntx) * kTZ;
  const int zend = min(z0 + kTZ, nzf - 1);
  const float* const src[3] = {in.fvx, in.fvz, in.fp};
  stage_tile<3>(sm, src, nzf, P, x0, z0);
  __syncthreads();
  const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
  const int ix = x0 + tx;
  if (ix < 3 || ix > nx - 4) return;
  const bool side = min(ix - 3, nx - 4 - ix) < C.npd;
  const int scol = side ? xstrip_col(ix, nx, C.npd) : 0;
  const float c = C.rk_c[s], w = (KIND == kStageLast) ? 0.f : C.rk_w[s];
#pragma unroll 1
  for (int j = 0; j < kRowsPerThread; ++j) {
    const int zr = ty + j * (kThreads / kTX);
    const int iz = z0 + zr;
    if (iz >= zend) break;
    FluidTile A;
    A.t = sm; A.r = zr + kHZ; A.c = tx + kHX;
    float ade[4] = {0.f, 0.f, 0.f, 0.f};
    const size_t si = (size_t)iz * C.Ps + scol;
    if (side) {
#pragma unroll
      for (int q = 0; q < 4; ++q) ade[q] = __ldg(in.fx[q] + si);
    }
    FluidK k = fluid_rhs<DIR>(C, A, iz, ix, side, ade);
    k.p += source_term(C, iz, ix, it, s);
    const size_t i = (size_t)iz * P + ix;
    rk_update<KIND>(k.vx, A.fvx(0, 0), un.fvx, out.fvx, acc.fvx, i, c, w);
    rk_update<KIND>(k.vz, A.fvz(0, 0), un.fvz, out.fvz, acc.fvz, i, c, w);
    rk_update<KIND>(k.p, A.fp(0, 0), un.fp, out.fp, acc.fp, i, c, w);
    if (side) {
      rk_update<KIND>(k.V0, ade[0], un.fx[0], out.fx[0], acc.fx[0], si, c, w);
      rk_update<KIND>(k.V1, ade[1], un.fx[1], out.fx[1], acc.fx[1], si, c, w);
      if (k.has_E) {
        rk_update<KIND>(k.E0, ade[2], un.fx[2], out.fx[2], acc.fx[2], si, c, w);
        rk_update<KIND>(k.E1, ade[3], un.fx[3], out.fx[3], acc.fx[3], si, c, w);
      }
    }
  }
}

template <int DIR, int KIND>
__device__ __forceinline__ void solid_tile(const Coef& C, const Fields& in, const Fields& out,
                                           const Fields& un, const Fields& acc, int s, int tile,
                                           int ntx, float* sm) {
  const int nx = C.nx, P = C.P, nzs = C.nzs, npd = C.npd;
  const int x0 = (tile % ntx) * kTX, z0 = 1 + (tile / ntx) * kTZ;
  const int zend = min(z0 + kTZ, nzs - 3);
  const float* const src[5] = {in.svx, in.svz, in.ssx, in.ssz, in.ssxz};
  stage_tile<5>(sm, src, nzs, P, x0, z0);
  __syncthreads();
  const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
  const int ix = x0 + tx;
  if (ix < 3 || ix > nx - 4) return;
  const bool side = min(ix - 3, nx - 4 - ix) < npd;
  const int scol = side ? xstrip_col(ix, nx, npd) : 0;
  const int zb0 = nzs - 3 - npd;  // first row of the bottom strip
  const float c = C.rk_c[s], w = (KIND == kStageLast) ? 0.f : C.rk_w[s];
#pragma unroll 1
  for (int j = 0; j < kRowsPerThread; ++j) {
    const int zr = ty + j * (kThreads / kTX);
    const int iz = z0 + zr;
    if (iz >= zend) break;
    const bool bottom = iz >= zb0;
    SolidTile A;
    A.t = sm; A.r = zr + kHZ; A.c = tx + kHX;
    float xade[4] = {0.f, 0.f, 0.f, 0.f}, zade[4] = {0.f, 0.f, 0.f, 0.f};
    const size_t sxi = (size_t)iz * C.Ps + scol;
    const size_t szi = (size_t)(iz - zb0) * P + ix;
    if (side) {
#pragma unroll
      for (int q = 0; q < 4; ++q) xade[q] = __ldg(in.sx[q] + sxi);
    }
    if (bottom) {
#pragma unroll
      for (int q = 0; q < 4; ++q) zade[q] = __ldg(in.sz[q] + szi);
    }
    SolidK k = solid_rhs<DIR>(C, A, iz, ix, side, bottom, xade, zade);
    const size_t i = (size_t)iz * P + ix;
    rk_update<KIND>(k.vx, A.svx(0, 0), un.svx, out.svx, acc.svx, i, c, w);
    rk_update<KIND>(k.vz, A.svz(0, 0), un.svz, out.svz, acc.svz, i, c, w);
    rk_update<KIND>(k.sx, A.ssx(0, 0), un.ssx, out.ssx, acc.ssx, i, c, w);
    rk_update<KIND>(k.sz, A.ssz(0, 0), un.ssz, out.ssz, acc.ssz, i, c, w);
    rk_update<KIND>(k.sxz, A.ssxz(0, 0), un.ssxz, out.ssxz, acc.ssxz, i, c, w);
    if (side) {
      rk_update<KIND>(k.XV0, xade[0], un.sx[0], out.sx[0], acc.sx[0], sxi, c, w);
      rk_update<KIND>(k.XV1, xade[1], un.sx[1], out.sx[1], acc.sx[1], sxi, c, w);
      rk_update<KIND>(k.XE0, xade[2], un.sx[2], out.sx[2], acc.sx[2], sxi, c, w);
      rk_update<KIND>(k.XE1, xade[3], un.sx[3], out.sx[3], acc.sx[3], sxi, c, w);
    }
    if (bottom) {
      rk_update<KIND>(k.ZV0, zade[0], un.sz[0], out.sz[0], acc.sz[0], szi, c, w);
      rk_update<KIND>(k.ZV1, zade[1], un.sz[1], out.sz[1], acc.sz[1], szi, c, w);
      rk_update<KIND>(k.ZE0, zade[2], un.sz[2], out.sz[2], acc.sz[2], szi, c, w);
      rk_update<KIND>(k.ZE1, zade[3], un.sz[3], out.sz[3], acc.sz[3], szi, c, w);
    }
  }
}

// Interface strip: fluid row nz_f-1 and solid row 0 of one column, their RHS,
// the normal/tangential coupling (pml_fs_kernels.cuh:754-827) and the RK update.
// In the last stage the eight coupled state values go to C.ipre, the filter's input.
template <int DIR, int KIND>
__device__ __forceinline__ void interface_strip(const Coef& C, const Fields& in, const Fields& out,
                                                const Fields& un, const Fields& acc, int s,
                                                int blk) {
  const int nx = C.nx, P = C.P, nzf = C.nzf, nzs = C.nzs, npd = C.npd;
  const int ix = blk * kThreads + threadIdx.x;
  if (ix < 3 || ix > nx - 4) return;
  const bool side = min(ix - 3, nx - 4 - ix) < npd;
  const int scol = side ? xstrip_col(ix, nx, npd) : 0;
  const int zb0 = nzs - 3 - npd;
  const bool bottom = 0 >= zb0;
  const float c = C.rk_c[s], w = (KIND == kStageLast) ? 0.f : C.rk_w[s];

  const size_t fi = (size_t)(nzf - 1) * P + ix;  // fluid interface cell
  const size_t si = ix;                          // solid interface cell
  FluidGlobal Af{in.fvx, in.fvz, in.fp, fi, P};
  SolidGlobal As{in.svx, in.svz, in.ssx, in.ssz, in.ssxz, si, P};
  float fade[4] = {0.f, 0.f, 0.f, 0.f}, xade[4] = {0.f, 0.f, 0.f, 0.f},
        zade[4] = {0.f, 0.f, 0.f, 0.f};
  const size_t fsi = (size_t)(nzf - 1) * C.Ps + scol, ssi = scol;
  const size_t szi = (size_t)(0 - zb0) * P + ix;
  if (side) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      fade[q] = __ldg(in.fx[q] + fsi);
      xade[q] = __ldg(in.sx[q] + ssi);
    }
  }
  if (bottom) {
#pragma unroll
    for (int q = 0; q < 4; ++q) zade[q] = __ldg(in.sz[q] + szi);
  }
  FluidK kf = fluid_rhs<DIR>(C, Af, nzf - 1, ix, side, fade);
  SolidK ks = solid_rhs<DIR>(C, As, 0, ix, side, bottom, xade, zade);

  // ---- coupling of the stage RHS on the interface ----
  const float2 n = __ldg(C.nrm + ix);
  const float vxf = kf.vx, vzf = kf.vz;
  float pf = kf.p;
  const float vxs = ks.vx, vzs = ks.vz, sxx = ks.sx, szz = ks.sz, sxz = ks.sxz;
  float vnf = n.x * vxf + n.y * vzf;
  const float vtf = n.y * vxf - n.x * vzf;
  float vns = n.x * vxs + n.y * vzs;
  const float vts = n.y * vxs - n.x * vzs;
  float snn = n.x * n.x * sxx + 2 * n.x * n.y * sxz + n.y * n.y * szz;
  float snt = n.x * n.y * (sxx - szz) + (n.y * n.y - n.x * n.x) * sxz;
  const float stt = n.y * n.y * sxx - 2 * n.x * n.y * sxz + n.x * n.x * szz;
  if (DIR == kDirF) {  // fluid takes the solid's normal velocity and traction
    vnf = vns;
    pf = -snn;
    snt = 0.f;
  } else {             // solid takes the fluid's
    vns = vnf;
    snn = -pf;
    snt = 0.f;
  }
  const float kv[8] = {n.x * vnf + n.y * vtf,
                       n.y * vnf - n.x * vtf,
                       pf,
                       n.x * vns + n.y * vts,
                       n.y * vns - n.x * vts,
                       n.x * n.x * snn + 2 * n.x * n.y * snt + n.y * n.y * stt,
                       n.y * n.y * snn - 2 * n.x * n.y * snt + n.x * n.x * stt,
                       -n.x * n.y * stt + (n.y * n.y - n.x * n.x) * snt};
  const float uin[8] = {Af.fvx(0, 0), Af.fvz(0, 0), Af.fp(0, 0), As.svx(0, 0),
                        As.svz(0, 0), As.ssx(0, 0), As.ssz(0, 0), As.ssxz(0, 0)};
  float* const outs[8] = {out.fvx, out.fvz, out.fp, out.svx, out.svz, out.ssx, out.ssz, out.ssxz};
  const float* const uns[8] = {un.fvx, un.fvz, un.fp, un.svx, un.svz, un.ssx, un.ssz, un.ssxz};
  float* const accs[8] = {acc.fvx, acc.fvz, acc.fp, acc.svx, acc.svz, acc.ssx, acc.ssz, acc.ssxz};
#pragma unroll
  for (int f = 0; f < 8; ++f) {
    const size_t i = f < 3 ? fi : si;
    if (KIND == kStageLast) {
      C.ipre[(size_t)f * P + ix] = fmaf(c, kv[f], accs[f][i]);
    } else {
      rk_update<KIND>(kv[f], uin[f], uns[f], outs[f], accs[f], i, c, w);
    }
  }
  if (side) {
    rk_update<KIND>(kf.V0, fade[0], un.fx[0], out.fx[0], acc.fx[0], fsi, c, w);
    rk_update<KIND>(kf.V1, fade[1], un.fx[1], out.fx[1], acc.fx[1], fsi, c, w);
    rk_update<KIND>(kf.E0, fade[2], un.fx[2], out.fx[2], acc.fx[2], fsi, c, w);
    rk_update<KIND>(kf.E1, fade[3], un.fx[3], out.fx[3], acc.fx[3], fsi, c, w);
    rk_update<KIND>(ks.XV0, xade[0], un.sx[0], out.sx[0], acc.sx[0], ssi, c, w);
    rk_update<KIND>(ks.XV1, xade[1], un.sx[1], out.sx[1], acc.sx[1], ssi, c, w);
    rk_update<KIND>(ks.XE0, xade[2], un.sx[2], out.sx[2], acc.sx[2], ssi, c, w);
    rk_update<KIND>(ks.XE1, xade[3], un.sx[3], out.sx[3], acc.sx[3], ssi, c, w);
  }
  if (bottom) {
    rk_update<KIND>(ks.ZV0, zade[0], un.sz[0], out.sz[0], acc.sz[0], szi, c, w);
    rk_update<KIND>(ks.ZV1, zade[1], un.sz[1], out.sz[1], acc.sz[1], szi, c, w);
    rk_update<KIND>(ks.ZE0, zade[2], un.sz[2], out.sz[2], acc.sz[2], szi, c, w);
    rk_update<KIND>(ks.ZE1, zade[3], un.sz[3], out.sz[3], acc.sz[3], szi, c, w);
  }
}

template <int DIR, int KIND>
__global__ void __launch_bounds__(kThreads)
    stage_kernel(Coef C, Fields in, Fields out, Fields un, Fields acc, int s, int ntx, int nbf,
                 int nbs) {
  extern __shared__ float4 smem_f4[];
  float* sm = reinterpret_cast<float*>(smem_f4);
  const int b = blockIdx.x;
  if (b < nbf) {
    const int it = __ldg(C.step);
    fluid_tile<DIR, KIND>(C, in, out, un, acc, s, it, b, ntx, sm);
  } else if (b < nbf + nbs) {
    solid_tile<DIR, KIND>(C, in, out, un, acc, s, b - nbf, ntx, sm);
  } else {
    interface_strip<DIR, KIND>(C, in, out, un, acc, s, b - nbf - nbs);
  }
}

// Post-step interface filter (7-point Gaussian along x, renormalised at the
// clamped ends) and continuity average (src/pml_fs_kernels.cu:428-525),
// evaluated out of place from C.ipre, so no block reads values another block
// already filtered. Then the receiver rows are sampled (src/main.cu:195-211)
// and the last block to finish advances the device step counter.
__global__ void __launch_bounds__(kThreads) finish_kernel(Coef C, Fields U) {
  const int nx = C.nx, P = C.P, nzf = C.nzf;
  const int ix = blockIdx.x * kThreads + threadIdx.x;
  const int it = *C.step;
  float r0 = 0.f, r1 = 0.f, r2 = 0.f;
  if (ix >= 3 && ix <= nx - 4) {
    const int klo = max(-3, 3 - ix), khi = min(3, nx - 4 - ix);
    float wsum = 0.0f;
    for (int k = klo; k <= khi; ++k) wsum += c_w7[k + 3];
    float v[8];
#pragma unroll
    for (int f = 0; f < 8; ++f) {
      float sum = 0.0f;
      for (int k = klo; k <= khi; ++k) sum += c_w7[k + 3] * C.ipre[(size_t)f * P + ix + k];
      v[f] = sum / wsum;
    }
    const float2 n = __ldg(C.nrm + ix);
    const float vnf = n.x * v[0] + n.y * v[1], vtf = n.y * v[0] - n.x * v[1];
    const float vns = n.x * v[3] + n.y * v[4], vts = n.y * v[3] - n.x * v[4];
    const float snn = n.x * n.x * v[5] + 2.0f * n.x * n.y * v[7] + n.y * n.y * v[6];
    const float stt = n.y * n.y * v[5] - 2.0f * n.x * n.y * v[7] + n.x * n.x * v[6];
    const float vn = 0.5f * (vnf + vns);
    const float sn = 0.5f * (snn - v[2]);
    const size_t fi = (size_t)(nzf - 1) * P + ix;
    U.fvx[fi] = n.x * vn + n.y * vtf;
    U.fvz[fi] = n.y * vn - n.x * vtf;
    U.fp[fi] = -sn;
    r0 = n.x * vn + n.y * vts;
    r1 = n.y * vn - n.x * vts;
    r2 = -sn;
    U.svx[ix] = r0;
    U.svz[ix] = r1;
    U.ssx[ix] = n.x * n.x * sn + n.y * n.y * stt;
    U.ssz[ix] = n.y * n.y * sn + n.x * n.x * stt;
    U.ssxz[ix] = n.x * n.y * (sn - stt);
    if (!(isfinite(r0) && isfinite(r1) && isfinite(r2))) atomicOr(C.status, 1);
  }
  if (ix < nx && C.rec != nullptr && C.gap > 0 && it % C.gap == 0) {
    const int j = it / C.gap;
    if (j < C.rec_cap) {
      float* row = C.rec + (size_t)j * 3 * nx;
      row[ix] = r0;
      row[nx + ix] = r1;
      row[2 * nx + ix] = r2;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(C.done, 1u);
    if (prev == gridDim.x - 1) {
      *C.done = 0u;
      *C.step = it + 1;
      __threadfence();
    }
  }
}

__global__ void set_step_kernel(int* step, unsigned* done, int it) {
  *step = it;
  *done = 0u;
}

// ---- host-side launchers ----------------------------------------------------

size_t stage_smem_bytes() { return size_t(5) * kTH * kTW * sizeof(float); }

void stage_grid(int nx, int nzf, int nzs, int* ntx, int* nbf, int* nbs, int* nbi) {
  *ntx = (nx + kTX - 1) / kTX;
  const int frows = nzf - 1 - 3;  // fluid rows 3..nz_f-2
  const int srows = nzs - 4;      // solid rows 1..nz_s-4
  *nbf = frows > 0 ? *ntx * ((frows + kTZ - 1) / kTZ) : 0;
  *nbs = srows > 0 ? *ntx * ((srows + kTZ - 1) / kTZ) : 0;
  *nbi = (nx + kThreads - 1) / kThreads;
}

template <int DIR, int KIND>
static cudaError_t launch_one(const Coef& C, const Fields& in, const Fields& out, const Fields& un,
                              const Fields& acc, int s, cudaStream_t st) {
  int ntx, nbf, nbs, nbi;
  stage_grid(C.nx, C.nzf, C.nzs, &ntx, &nbf, &nbs, &nbi);
  const size_t smem = stage_smem_bytes();
  stage_kernel<DIR, KIND><<<nbf + nbs + nbi, kThreads, smem, st>>>(C, in, out, un, acc, s, ntx,
                                                                   nbf, nbs);
  return cudaGetLastError();
}

template <int DIR, int KIND>
static cudaError_t configure_one() {
  return cudaFuncSetAttribute(stage_kernel<DIR, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)stage_smem_bytes());
}

cudaError_t configure_device() {
  cudaError_t e;
  if ((e = configure_one<kDirF, kStageFirst>()) != cudaSuccess) return e;
  if ((e = configure_one<kDirF, kStageMid>()) != cudaSuccess) return e;
  if ((e = configure_one<kDirF, kStageLast>()) != cudaSuccess) return e;
  if ((e = configure_one<kDirB, kStageFirst>()) != cudaSuccess) return e;
  if ((e = configure_one<kDirB, kStageMid>()) != cudaSuccess) return e;
  return configure_one<kDirB, kStageLast>();
}

cudaError_t launch_stage(const Coef& C, const Fields& in, const Fields& out, const Fields& un,
                         const Fields& acc, int stage, int dir, cudaStream_t st) {
  const int kind = stage == 0 ? kStageFirst : (stage == 3 ? kStageLast : kStageMid);
  if (dir == kDirF) {
    if (kind == kStageFirst) return launch_one<kDirF, kStageFirst>(C, in, out, un, acc, stage, st);
    if (kind == kStageMid) return launch_one<kDirF, kStageMid>(C, in, out, un, acc, stage, st);
    return launch_one<kDirF, kStageLast>(C, in, out, un, acc, stage, st);
  }
  if (kind == kStageFirst) return launch_one<kDirB, kStageFirst>(C, in, out, un, acc, stage, st);
  if (kind == kStageMid) return launch_one<kDirB, kStageMid>(C, in, out, un, acc, stage, st);
  return launch_one<kDirB, kStageLast>(C, in, out, un, acc, stage, st);
}

cudaError_t launch_finish(const Coef& C, const Fields& U, cudaStream_t st) {
  const int nb = (C.nx + kThreads - 1) / kThreads;
  finish_kernel<<<nb, kThreads, 0, st>>>(C, U);
  return cudaGetLastError();
}

cudaError_t launch_set_step(const Coef& C, int it, cudaStream_t st) {
  set_step_kernel<<<1, 1, 0, st>>>(C.step, C.done, it);
  return cudaGetLastError();
}

cudaError_t upload_constants(const float* srcw25, const float* w7) {
  cudaError_t e = cudaMemcpyToSymbol(c_srcw, srcw25, 25 * sizeof(float));
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_w7, w7, 7 * sizeof(float));
}

}  // namespace mfdm
