// sm_100a kernels of the solid-only time step with a free surface (see mfdm_solid.h),
// and of its four-side CFS-PML variant (the CPML instantiations below).
//
// One launch per RK stage does the whole stage: velocity and stress
// right-hand sides of every cell (the reference's update_velocity and
// update_stress, which run as two kernels on two streams), the free-surface
// ghost fluxes (built on the fly from the stage input instead of a separate
// build_ghost_flux launch), the explosive source and the fused RK4 update
// (the reference's vector_add / vector_self_add launches over full grids).
// A fifth launch per step samples the receiver row and advances the device
// step counter. Each block stages the five stage-input fields of its 32x16
// cells and their 3-cell halo in shared memory with independent float4 loads
// (all in flight at once, together with the point-wise operands of every
// thread's first row), then every thread computes two rows from shared memory;
// coefficients, ADE memory and the RK operands are point-wise global reads,
// all of a row's issued before its arithmetic and its stores.
#include "mfdm_device.cuh"
#include "mfdm_solid.h"

namespace mfdm {
namespace solid {
namespace {

constexpr int kBX = 32, kBY = 8;
#ifndef MFDM_SOLID_ROWS
#define MFDM_SOLID_ROWS 16
#endif
constexpr int kTZ = MFDM_SOLID_ROWS;  // rows per block (kTZ / kBY per thread)
static_assert(kTZ % kBY == 0 && 5 * (kTZ + 6) * (kBX + 8) * 4 <= 48 * 1024, "tile rows");
constexpr int kHW = kBX + 8;     // tile row: columns c0 .. c0 + 39, c0 = first cell - 3
constexpr int kHH = kTZ + 6;     // tile rows: r0 .. r0 + kTZ + 5, r0 = first row - 3
enum { kVX = 0, kVZ, kSX, kSZ, kSXZ };

// The 5x5 weights of the explosive source (src/elements.cu:34-40).
__constant__ float kSrcW[25] = {0.0030f, 0.0133f, 0.0219f, 0.0133f, 0.0030f, 0.0133f, 0.0596f,
                                0.0983f, 0.0596f, 0.0133f, 0.0219f, 0.0983f, 0.1621f, 0.0983f,
                                0.0219f, 0.0133f, 0.0596f, 0.0983f, 0.0596f, 0.0133f, 0.0030f,
                                0.0133f, 0.0219f, 0.0133f, 0.0030f};
// Point-wise coefficients of a cell, in this order.
enum { kCXIX = 0, kCXIZ, kCZEX, kCZEZ, kCRR, kC11, kC13, kC33, kC55, kNCoef };

struct Out {
  float vx, vz, sx, sz, sxz;
  float XV0, XV1, XE0, XE1, ZV0, ZV1, ZE0, ZE1;
};

// Zeta-ADE row of a cell in a zeta-PML band: the bottom band (rows
// nz-3-npd..nz-4) at 0..npd-1; with CPML the top band (rows 3..npd+2) after it.
template <bool CPML>
__device__ __forceinline__ int zeta_row(int iz, int nz, int npd) {
  if (CPML && iz <= npd + 2) return npd + iz - 3;
  return iz - (nz - 3 - npd);
}

// Right-hand side of cell (iz, ix), 3 <= iz <= nz-4 (include/pml_fs_kernels.cuh:10-307).
// CPML: the four-side variant Cpml::SolidOnly (include/cpml_kernels.cuh:8-217):
// no free surface, so every row takes the plain biased operators (rows 0..2
// are zero), and the zeta-PML also covers the top band (rows 3..npd+2).
// `A(q, dz, dx)` returns stage-input field q (kVX..kSXZ) dz rows and dx columns
// away, |dz|, |dx| <= 3; the ADE memory of S is read from global memory.
// IN: the caller guarantees a cell at least three rows below the free surface
// and outside every absorbing strip (the branch-free body of interior blocks).
// `K(c)` returns point-wise coefficient c (kCXIX..kC55) of the cell.
template <int DIR, bool IN, bool CPML, class Acc, class Kc>
__device__ __forceinline__ Out rhs(const SCoef& C, const SFields& S, const Acc& A, const Kc& K,
                                   int iz, int ix) {
  Out o;
  const int P = C.P, nx = C.nx, nz = C.nz, npd = C.npd;
  const size_t i = (size_t)iz * P + ix;
  const int dist = (IN || CPML) ? 3 : iz - 3, distx = min(ix - 3, nx - 4 - ix);
  const bool side = !IN && distx < npd;
  const bool bottom = !IN && (iz >= nz - 3 - npd || (CPML && iz <= npd + 2));
  const int scol = side ? xstrip_col(ix, nx, npd) : 0;
  const size_t si = (size_t)iz * C.Ps + scol, zi = (size_t)zeta_row<CPML>(iz, nz, npd) * P + ix;
  const float xix = K(kCXIX), xiz = K(kCXIZ), zex = K(kCZEX), zez = K(kCZEZ);
  const float gxixi = xix * xix + xiz * xiz, gzeze = zex * zex + zez * zez;
  const float gxize = xix * zex + xiz * zez;
  auto dx5 = [&](int q) {
    return d5<DIR>(A(q, 0, -3), A(q, 0, -2), A(q, 0, -1), A(q, 0, 0), A(q, 0, 1), A(q, 0, 2),
                   A(q, 0, 3));
  };
  auto dzn = [&](int q, int d) {
    auto col = [&](int j) { return A(q, j, 0); };
    return dz_near<DIR>(col, d, true);
  };
  o.XV0 = o.XV1 = o.XE0 = o.XE1 = o.ZV0 = o.ZV1 = o.ZE0 = o.ZE1 = 0.f;

  // ---- momentum: rho dv/dt = div sigma ----
  {
    float rvx, rvz, dxx = 0.f, dxz = 0.f, dzx = 0.f, dzz = 0.f;
    if (!IN && dist < 3) {
      // conservative rows under the free surface; above it the image G = -F of
      // the rows below (src/pml_fs_kernels.cu:7-19)
      auto Fs = [&](int r) -> float2 {
        const size_t k = (size_t)r * P + ix;
        const float Jk = __ldg(C.J + k), ax = __ldg(C.zex + k), az = __ldg(C.zez + k);
        const float sx = A(kSX, r - iz, 0), sz = A(kSZ, r - iz, 0), sxz = A(kSXZ, r - iz, 0);
        return make_float2(Jk * (ax * sx + az * sxz), Jk * (ax * sxz + az * sz));
      };
      auto Fxi = [&](int j) -> float2 {
        const size_t k = i + j;
        const float Jk = __ldg(C.J + k), ax = __ldg(C.xix + k), az = __ldg(C.xiz + k);
        const float sx = A(kSX, 0, j), sz = A(kSZ, 0, j), sxz = A(kSXZ, 0, j);
        return make_float2(Jk * (ax * sx + az * sxz), Jk * (ax * sxz + az * sz));
      };
      auto Fze = [&](int j) -> float2 {
        const int r = iz + j;
        if (r >= 3) return Fs(r);
        const float2 b = Fs(6 - r);
        return make_float2(-b.x, -b.y);
      };
      const float2 a = dflux<DIR>(Fxi), b = dflux<DIR>(Fze);
      const float Jc = __ldg(C.J + i);
      rvx = (a.x + b.x) / Jc;
      rvz = (a.y + b.y) / Jc;
      const float dxsx = dx5(kSX), dxsz = dx5(kSZ), dxsxz = dx5(kSXZ);
      const float dzsx = dzn(kSX, dist), dzsz = dzn(kSZ, dist), dzsxz = dzn(kSXZ, dist);
      dxx = xix * (dxsx + gxize / gxixi * dzsx) + xiz * (dxsxz + gxize / gxixi * dzsxz);
      dxz = xix * (dxsxz + gxize / gxixi * dzsxz) + xiz * (dxsz + gxize / gxixi * dzsz);
    } else {
      const float sxdx = dx5(kSX), sxdz = dzn(kSX, 3), szdx = dx5(kSZ), szdz = dzn(kSZ, 3);
      const float tdx = dx5(kSXZ), tdz = dzn(kSXZ, 3);
      rvx = xix * sxdx + zex * sxdz + xiz * tdx + zez * tdz;
      rvz = xix * tdx + zex * tdz + xiz * szdx + zez * szdz;
      if (side || bottom) {
        dxx = xix * (sxdx + gxize / gxixi * sxdz) + xiz * (tdx + gxize / gxixi * tdz);
        dxz = xix * (tdx + gxize / gxixi * tdz) + xiz * (szdx + gxize / gxixi * szdz);
        dzx = zex * (sxdz + gxize / gzeze * sxdx) + zez * (gxize / gzeze * tdx + tdz);
        dzz = zex * (gxize / gzeze * tdx + tdz) + zez * (gxize / gzeze * szdx + szdz);
      }
    }
    const float ir = K(kCRR);
    o.vx = rvx * ir;
    o.vz = rvz * ir;
    if (side) {
      const float4 p = __ldg(C.pmlx + ix);
      const float V0 = __ldg(S.x[0] + si), V1 = __ldg(S.x[1] + si);
      o.XV0 = -p.y * V0 + p.x * dxx;
      o.XV1 = -p.y * V1 + p.x * dxz;
      o.vx += ((p.z - 1.0f) * dxx - p.z * V0) * ir;
      o.vz += ((p.z - 1.0f) * dxz - p.z * V1) * ir;
    }
    if (bottom) {
      const float4 p = __ldg(C.pmlz + iz);
      const float V0 = __ldg(S.z[0] + zi), V1 = __ldg(S.z[1] + zi);
      o.ZV0 = -p.y * V0 + p.x * dzx;
      o.ZV1 = -p.y * V1 + p.x * dzz;
      o.vx += ((p.z - 1.0f) * dzx - p.z * V0) * ir;
      o.vz += ((p.z - 1.0f) * dzz - p.z * V1) * ir;
    }
  }
  // ---- stress ----
  {
    const float c11 = K(kC11), c13 = K(kC13), c33 = K(kC33), c55 = K(kC55);
    const float dvx_dxi = dx5(kVX), dvz_dxi = dx5(kVZ);
    if (!IN && dist == 0) {
      // traction-free row: the zeta derivatives eliminated through the ALM
      // coefficients (src/elements.cu:907-977)
      const float a0 = __ldg(C.alm + ix), a1 = __ldg(C.alm + P + ix), a2 = __ldg(C.alm + 2 * P + ix),
                  a3 = __ldg(C.alm + 3 * P + ix), a4 = __ldg(C.alm + 4 * P + ix),
                  a5 = __ldg(C.alm + 5 * P + ix);
      o.sx = (c11 * a0 + c13 * a1) * dvx_dxi + (c11 * a3 + c13 * a4) * dvz_dxi;
      o.sz = (c13 * a0 + c33 * a1) * dvx_dxi + (c13 * a3 + c33 * a4) * dvz_dxi;
      o.sxz = c55 * (a2 * dvx_dxi + a5 * dvz_dxi);
      if (side) {
        const float4 p = __ldg(C.pmlx + ix);
        const float E0 = __ldg(S.x[2] + si), E1 = __ldg(S.x[3] + si);
        o.XE0 = -p.y * E0 + p.x * dvx_dxi;
        o.XE1 = -p.y * E1 + p.x * dvz_dxi;
        const float cxx_x = c11 * a0 + c13 * a1, cxx_z = c11 * a3 + c13 * a4;
        o.sx += (p.z - 1.0f) * (cxx_x * dvx_dxi + cxx_z * dvz_dxi) - p.z * (cxx_x * E0 + cxx_z * E1);
        const float czz_x = c13 * a0 + c33 * a1, czz_z = c13 * a3 + c33 * a4;
        o.sz += (p.z - 1.0f) * (czz_x * dvx_dxi + czz_z * dvz_dxi) - p.z * (czz_x * E0 + czz_z * E1);
        o.sxz += c55 * ((p.z - 1.0f) * (a2 * dvx_dxi + a5 * dvz_dxi) - p.z * (a2 * E0 + a5 * E1));
      }
      return o;
    }
    const float dvx_dze = dzn(kVX, dist), dvz_dze = dzn(kVZ, dist);
    o.sx = c11 * (xix * dvx_dxi + zex * dvx_dze) + c13 * (xiz * dvz_dxi + zez * dvz_dze);
    o.sz = c13 * (xix * dvx_dxi + zex * dvx_dze) + c33 * (xiz * dvz_dxi + zez * dvz_dze);
    o.sxz = c55 * (xiz * dvx_dxi + zez * dvx_dze + xix * dvz_dxi + zex * dvz_dze);
    if (side) {
      const float Dvx = dvx_dxi + (gxize / gxixi) * dvx_dze, Dvz = dvz_dxi + (gxize / gxixi) * dvz_dze;
      const float4 p = __ldg(C.pmlx + ix);
      const float E0 = __ldg(S.x[2] + si), E1 = __ldg(S.x[3] + si), invb = p.z;
      o.XE0 = -p.y * E0 + p.x * Dvx;
      o.XE1 = -p.y * E1 + p.x * Dvz;
      o.sx += c11 * (invb - 1.0f) * xix * Dvx + c13 * (invb - 1.0f) * xiz * Dvz -
              invb * c11 * xix * E0 - invb * c13 * xiz * E1;
      o.sz += c13 * (invb - 1.0f) * xix * Dvx + c33 * (invb - 1.0f) * xiz * Dvz -
              invb * c13 * xix * E0 - invb * c33 * xiz * E1;
      o.sxz += c55 * (invb - 1.0f) * (xiz * Dvx + xix * Dvz) - invb * c55 * xiz * E0 -
               invb * c55 * xix * E1;
    }
    if (bottom) {
      const float Dvx = dvx_dze + (gxize / gzeze) * dvx_dxi, Dvz = dvz_dze + (gxize / gzeze) * dvz_dxi;
      const float4 p = __ldg(C.pmlz + iz);
      const float E0 = __ldg(S.z[2] + zi), E1 = __ldg(S.z[3] + zi), invb = p.z;
      o.ZE0 = -p.y * E0 + p.x * Dvx;
      o.ZE1 = -p.y * E1 + p.x * Dvz;
      o.sx += c11 * (invb - 1.0f) * zex * Dvx + c13 * (invb - 1.0f) * zez * Dvz -
              invb * c11 * zex * E0 - invb * c13 * zez * E1;
      o.sz += c13 * (invb - 1.0f) * zex * Dvx + c33 * (invb - 1.0f) * zez * Dvz -
              invb * c13 * zex * E0 - invb * c33 * zez * E1;
      o.sxz += c55 * (invb - 1.0f) * (zez * Dvx + zex * Dvz) - invb * c55 * zez * E0 -
               invb * c55 * zex * E1;
    }
  }
  return o;
}

template <int KIND>
__device__ __forceinline__ void upd(float k, const float* in, const float* un, float* out,
                                    float* acc, size_t i, float c, float w) {
  rk_update<KIND>(k, KIND == kStageFirst ? __ldg(in + i) : 0.f, un, out, acc, i, c, w);
}

// The point-wise operands of one cell: U^n (`u`, the stage input itself at
// stage 0, taken from the tile), the accumulator (`a`) and the coefficients
// (`k`). They are loaded into registers before any store of the row -- the
// first row's before the tile barrier, so that their DRAM round trips overlap
// the tile load (the output and accumulator pointers may alias the inputs as
// far as the compiler knows, which would otherwise order each field's loads
// after the previous field's stores). Loading the next row's under the
// current row's arithmetic needs 80 registers and was slower.
struct Pt { float u[5], a[5], k[kNCoef]; };

template <int KIND>
__device__ __forceinline__ void load_pt(Pt& p, const SCoef& C, const SFields& un,
                                        const SFields& acc, size_t i) {
  const float* const pu[5] = {un.vx, un.vz, un.sx, un.sz, un.sxz};
  const float* const pa[5] = {acc.vx, acc.vz, acc.sx, acc.sz, acc.sxz};
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    if (KIND == kStageMid) p.u[q] = __ldg(pu[q] + i);
    if (KIND != kStageFirst) p.a[q] = pa[q][i];
  }
  p.k[kCXIX] = __ldg(C.xix + i);
  p.k[kCXIZ] = __ldg(C.xiz + i);
  p.k[kCZEX] = __ldg(C.zex + i);
  p.k[kCZEZ] = __ldg(C.zez + i);
  p.k[kCRR] = __ldg(C.rcp_rho + i);
  p.k[kC11] = __ldg(C.C11 + i);
  p.k[kC13] = __ldg(C.C13 + i);
  p.k[kC33] = __ldg(C.C33 + i);
  p.k[kC55] = __ldg(C.C55 + i);
}

template <int KIND>
__device__ __forceinline__ void store5(const Out& o, const Pt& r, const SFields& out,
                                       const SFields& acc, size_t i, float c, float w) {
  float* const po[5] = {out.vx, out.vz, out.sx, out.sz, out.sxz};
  float* const pa[5] = {acc.vx, acc.vz, acc.sx, acc.sz, acc.sxz};
  const float k[5] = {o.vx, o.vz, o.sx, o.sz, o.sxz};
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    if (KIND == kStageFirst) {
      po[q][i] = fmaf(c, k[q], r.u[q]);
      pa[q][i] = fmaf(w, k[q], r.u[q]);
    } else if (KIND == kStageMid) {
      po[q][i] = fmaf(c, k[q], r.u[q]);
      pa[q][i] = fmaf(w, k[q], r.a[q]);
    } else {
      po[q][i] = fmaf(c, k[q], r.a[q]);
    }
  }
}

// The kTZ / kBY rows of column ix owned by this thread, from the staged tile;
// `p` holds the first row's point-wise operands on entry.
template <int DIR, int KIND, bool IN, bool CPML>
__device__ __forceinline__ void rows(const SCoef& C, const SFields& in, const SFields& out,
                                     const SFields& un, const SFields& acc,
                                     const float (&tile)[5][kHH][kHW], int r0, int ix, int s,
                                     float c, float w, Pt& p) {
  const int nx = C.nx, nz = C.nz, npd = C.npd, P = C.P;
  const int it = IN ? 0 : __ldg(C.step);
#pragma unroll 1
  for (int k = 0; k < kTZ / kBY; ++k) {
    const int lz = 3 + threadIdx.y + k * kBY, iz = r0 + lz;
    if (iz > nz - 4) return;
    auto A = [&](int q, int dz, int dx) { return tile[q][lz + dz][3 + threadIdx.x + dx]; };
    const size_t i = (size_t)iz * P + ix;
    if (k > 0) load_pt<KIND>(p, C, un, acc, i);
    if (KIND == kStageFirst) {
#pragma unroll
      for (int q = 0; q < 5; ++q) p.u[q] = A(q, 0, 0);
    }
    auto K = [&](int cf) { return p.k[cf]; };
    Out o = rhs<DIR, IN, CPML>(C, in, A, K, iz, ix);
    if (!IN) {
      // explosive source on both normal stresses (src/pml_fs_kernels.cu:22-26)
      const int sx = ix - C.srcx, sz = iz - C.srcz;
      if (C.srcx >= 0 && sx >= -2 && sx <= 2 && sz >= -2 && sz <= 2 && it >= 0 && it < C.src_steps) {
        const float q = __ldg(C.src_amp + (size_t)it * 4 + s) * kSrcW[(sz + 2) * 5 + (sx + 2)];
        o.sx += q;
        o.sz += q;
      }
    }
    store5<KIND>(o, p, out, acc, i, c, w);
    if (!IN && min(ix - 3, nx - 4 - ix) < npd) {
      const size_t si = (size_t)iz * C.Ps + xstrip_col(ix, nx, npd);
      upd<KIND>(o.XV0, in.x[0], un.x[0], out.x[0], acc.x[0], si, c, w);
      upd<KIND>(o.XV1, in.x[1], un.x[1], out.x[1], acc.x[1], si, c, w);
      upd<KIND>(o.XE0, in.x[2], un.x[2], out.x[2], acc.x[2], si, c, w);
      upd<KIND>(o.XE1, in.x[3], un.x[3], out.x[3], acc.x[3], si, c, w);
    }
    if (!IN && (iz >= nz - 3 - npd || (CPML && iz <= npd + 2))) {
      const size_t zi = (size_t)zeta_row<CPML>(iz, nz, npd) * P + ix;
      upd<KIND>(o.ZV0, in.z[0], un.z[0], out.z[0], acc.z[0], zi, c, w);
      upd<KIND>(o.ZV1, in.z[1], un.z[1], out.z[1], acc.z[1], zi, c, w);
      upd<KIND>(o.ZE0, in.z[2], un.z[2], out.z[2], acc.z[2], zi, c, w);
      upd<KIND>(o.ZE1, in.z[3], un.z[3], out.z[3], acc.z[3], zi, c, w);
    }
  }
}

template <int DIR, int KIND, bool CPML>
__global__ void __launch_bounds__(kBX * kBY, 4) k_stage(SCoef C, SFields in, SFields out,
                                                                      SFields un, SFields acc, int s,
                                                                      float c, float w) {
  __shared__ __align__(16) float tile[5][kHH][kHW];
  const int nx = C.nx, nz = C.nz, npd = C.npd, P = C.P;
  const int c0 = blockIdx.x * kBX, r0 = blockIdx.y * kTZ;
  const int ix = 3 + c0 + threadIdx.x, iz0 = r0 + 3 + threadIdx.y;
  // the first row's point-wise operands, in flight together with the tile
  Pt p;
  if (ix <= nx - 4 && iz0 <= nz - 4) load_pt<KIND>(p, C, un, acc, (size_t)iz0 * P + ix);
  // Stage the tile: rows r0.. (below nz), float4 columns c0.. (below P; the
  // pitch is a multiple of 32 floats, so every float4 lies in one row and no
  // column at or beyond nx is ever read back). 250 of the 256 threads each own
  // one float4 column of every 25th tile row.
  {
    constexpr int kV = kHW / 4, kRowsPerPass = (kBX * kBY) / kV;
    const int tid = threadIdx.y * kBX + threadIdx.x, vr = tid / kV, vc = (tid - vr * kV) * 4;
    if (vr < kRowsPerPass && c0 + vc < P) {
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        const float* f = q == kVX ? in.vx : q == kVZ ? in.vz : q == kSX ? in.sx : q == kSZ ? in.sz : in.sxz;
#pragma unroll
        for (int rr = vr; rr < kHH; rr += kRowsPerPass)
          if (r0 + rr < nz)
            *reinterpret_cast<float4*>(&tile[q][rr][vc]) =
                __ldg(reinterpret_cast<const float4*>(f + (size_t)(r0 + rr) * P + c0 + vc));
      }
    }
  }
  __syncthreads();
  if (ix > nx - 4) return;
  // Blocks whose cells are all at least three rows below the free surface (with
  // CPML: below the top band), in no absorbing strip and away from the source
  // take the branch-free body.
  const bool interior = r0 >= (CPML ? npd : 3) && r0 + kTZ + 2 < nz - 3 - npd && c0 >= npd &&
                        c0 + kBX + 2 <= nx - 4 - npd &&
                        (C.srcx < 0 || C.srcx + 2 < c0 + 3 || C.srcx - 2 > c0 + kBX + 2 ||
                         C.srcz + 2 < r0 + 3 || C.srcz - 2 > r0 + kTZ + 2);
  if (interior)
    rows<DIR, KIND, true, CPML>(C, in, out, un, acc, tile, r0, ix, s, c, w, p);
  else
    rows<DIR, KIND, false, CPML>(C, in, out, un, acc, tile, r0, ix, s, c, w, p);
}

__global__ void k_finish(SCoef C, SFields U) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int it = *C.step;
  if (ix < C.nx) {
    const float v = U.vz[(size_t)C.rec_row * C.P + ix];
    if (!isfinite(v)) atomicOr(C.status, 1);
    if (C.rec != nullptr && C.gap > 0 && it % C.gap == 0) {
      const int j = it / C.gap;
      if (j < C.rec_cap) C.rec[(size_t)j * C.nx + ix] = v;
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

__global__ void k_set_step(int* step, unsigned* done, int it) {
  *step = it;
  *done = 0u;
}

template <int DIR, int KIND>
cudaError_t launch_t(const SCoef& C, const SFields& in, const SFields& out, const SFields& un,
                     const SFields& acc, int s, cudaStream_t st) {
  const dim3 grid(unsigned((C.nx - 6 + kBX - 1) / kBX), unsigned((C.nz - 6 + kTZ - 1) / kTZ));
  const float c = C.rk_c[s], w = KIND == kStageLast ? 0.f : C.rk_w[s];
  if (C.cpml)
    k_stage<DIR, KIND, true><<<grid, dim3(kBX, kBY), 0, st>>>(C, in, out, un, acc, s, c, w);
  else
    k_stage<DIR, KIND, false><<<grid, dim3(kBX, kBY), 0, st>>>(C, in, out, un, acc, s, c, w);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_stage(const SCoef& C, const SFields& in, const SFields& out, const SFields& un,
                         const SFields& acc, int stage, int dir, cudaStream_t st) {
  if (dir == kDirF) {
    if (stage == 0) return launch_t<kDirF, kStageFirst>(C, in, out, un, acc, stage, st);
    if (stage == 3) return launch_t<kDirF, kStageLast>(C, in, out, un, acc, stage, st);
    return launch_t<kDirF, kStageMid>(C, in, out, un, acc, stage, st);
  }
  if (stage == 0) return launch_t<kDirB, kStageFirst>(C, in, out, un, acc, stage, st);
  if (stage == 3) return launch_t<kDirB, kStageLast>(C, in, out, un, acc, stage, st);
  return launch_t<kDirB, kStageMid>(C, in, out, un, acc, stage, st);
}

cudaError_t launch_finish(const SCoef& C, const SFields& U, cudaStream_t st) {
  k_finish<<<unsigned((C.nx + 255) / 256), 256, 0, st>>>(C, U);
  return cudaGetLastError();
}

cudaError_t launch_set_step(const SCoef& C, int it, cudaStream_t st) {
  k_set_step<<<1, 1, 0, st>>>(C.step, C.done, it);
  return cudaGetLastError();
}

}  // namespace solid
}  // namespace mfdm
