// Device-side building blocks of the fluid-solid time step: stencil operators,
// per-cell right-hand sides, interface coupling and the RK4 stage update.
//
// Layout in HBM (all FP32, row-major, x fastest, row pitch P floats, P a
// multiple of 32 so every row starts on a 128-byte boundary):
//   fluid fields  vx, vz, p              [nz_f][P]
//   solid fields  vx, vz, sx, sz, sxz    [nz_s][P]
//   metric        J, xi_x, xi_z, ze_x, ze_z over global rows [nz_f+nz_s-1][P]
//                 (fluid row r = global row r; solid row r = global row r+nz_f-1)
//   ADE memory    fluid xi strips [nz_f][Ps], solid xi strips [nz_s][Ps]
//                 (left columns 3..2+npd then right columns nx-3-npd..nx-4),
//                 solid zeta strip [npd][P] (solid rows nz_s-3-npd..nz_s-4).
// The reference keeps ADE memory over the full grid (src/elements.cu:737-758);
// only the strip cells are ever non-zero, so only those are stored here.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mfdm {

// Geometry of the streaming stage kernel, shared with the host (tensor-map boxes).
constexpr int kStageTX = 64;             // computed columns per strip
constexpr int kStageSW = kStageTX + 8;   // staged stencil row width (4-column halo each side)
constexpr int kStageR = 4;               // rows per chunk

// TMA descriptors of one stage launch. Each maps a block [field][rows][P] of
// one RK set (fluid: vx, vz, p; solid: vx, vz, sx, sz, sxz) or of the
// coefficients (fluid: xi_x, xi_z, ze_x, ze_z, rho, K; solid: xi_x, xi_z,
// ze_x, ze_z, rho, C11, C13, C33, C55); one box = all fields of kStageR rows.
// Stage-input boxes land as [row][field][col], the others as [field][row][col].
// The state maps have a fourth dimension, the shot; the coefficient maps none.
struct StageMaps {
  CUtensorMap fin, sin;    // stage input, box {kStageSW, nfield, kStageR}
  CUtensorMap fun, sun;    // U^n, box {kStageTX, kStageR, nfield}
  CUtensorMap facc, sacc;  // accumulator, box {kStageTX, kStageR, nfield}
  CUtensorMap fcoef, scoef;  // coefficients, box {kStageTX, kStageR, 6 | 9}
};

// DRP-optimised biased 5-point first derivative (reference include/tools_func.cuh:6-10).
// The literals sum to -6e-5, not 0: they are kept exactly.
constexpr float kAm1 = -0.30874f;
constexpr float kA0 = -0.63260f;
constexpr float kA1 = +1.23300f;
constexpr float kA2 = -0.33340f;
constexpr float kA3 = +0.04168f;
// One-sided 4-2 and 2-2 operators near boundaries (include/tools_func.cuh:12-17).
constexpr float kM42_0 = -7.0f / 6.0f;
constexpr float kM42_1 = +8.0f / 6.0f;
constexpr float kM42_2 = -1.0f / 6.0f;

enum { kDirF = 0, kDirB = 1 };
enum { kStageFirst = 0, kStageMid = 1, kStageLast = 2 };

// Everything a stage kernel needs besides the four RK state sets.
struct Coef {
  int nx, nzf, nzs, P, npd, Ps;
  const float* __restrict__ K;     // fluid bulk modulus [nz_f][P]
  const float* __restrict__ rhof;  // fluid density
  const float* __restrict__ C11;   // solid stiffness [nz_s][P]
  const float* __restrict__ C13;
  const float* __restrict__ C33;
  const float* __restrict__ C55;
  const float* __restrict__ rhos;  // solid density
  const float* __restrict__ J;     // metric, global rows
  const float* __restrict__ xix;
  const float* __restrict__ xiz;
  const float* __restrict__ zex;
  const float* __restrict__ zez;
  const float4* __restrict__ pmlx;  // per column: d/beta, alpha + d/beta, 1/beta
  const float4* __restrict__ pmlz;  // per solid row (zeta strip)
  const float4* __restrict__ pmlzf; // per fluid row (top zeta band, four-side CPML only)
  int cpml;                         // 1: CFS-PML on all four sides (Cpml::FluidSolid, the
                                    // CPML kernel instantiations), 0: free surface on top
  const float2* __restrict__ nrm;   // interface unit normal per column
  const float* __restrict__ src_amp;  // Ricker value per (step, stage): [steps][4]
  int src_steps;                    // steps the table holds
  int src_it0;                      // time index of the table's first row (0: absolute)
  int srcx, srcz;                   // source column / fluid row (srcx < 0: none)
  float rk_c[4];                    // dt/2, dt/2, dt, dt/6
  float rk_w[3];                    // dt/6, dt/3, dt/3
  int gap;                          // record interval in steps
  int rec_cap;                      // record ring capacity in samples
  float* rec;                       // [rec_cap][3][nx]: solid vx, solid vz, fluid p
  int* step;                        // device step counter (time index of the running step)
  unsigned* done;                   // block arrival counter of the finish kernel
  float* ipre;                      // interface rows before the filter [8][P]
  int* status;                      // sticky error word (non-finite detector)
  int seg;                          // rows per segment block of the stage launches (0: 24)
  int variant;                      // stage kernel build: 2 or 3 blocks per SM (0: by grid size)
  // Shots stepped together (the stage launch's fastest block index, blockIdx.y
  // of the finish kernel). Every per-shot
  // buffer of shot b sits b strides after shot 0's: the RK sets, ADE strips,
  // PML tables and interface rows (shot_stride), the Ricker table (src_stride)
  // and the receiver rows (rec_stride), all in floats.
  int nshots;
  size_t shot_stride, src_stride, rec_stride;
  const int2* __restrict__ src_pos;  // per-shot source (x, z); nullptr: srcx, srcz
};

// One RK4 state set (state, stage ping/pong or accumulator).
struct Fields {
  float* fvx; float* fvz; float* fp;
  float* svx; float* svz; float* ssx; float* ssz; float* ssxz;
  float* fx[4];  // fluid xi ADE: Vx, Vz, Ex, Ez
  float* sx[4];  // solid xi ADE
  float* sz[4];  // solid zeta ADE
  float* fz[4];  // fluid zeta ADE, top band rows 3..npd+2 [npd][P] (four-side CPML only)
};

// The set of one shot: every pointer `so` floats further.
__device__ __forceinline__ Fields shot_fields(const Fields& f, size_t so) {
  Fields g;
  g.fvx = f.fvx + so; g.fvz = f.fvz + so; g.fp = f.fp + so;
  g.svx = f.svx + so; g.svz = f.svz + so; g.ssx = f.ssx + so; g.ssz = f.ssz + so;
  g.ssxz = f.ssxz + so;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    g.fx[q] = f.fx[q] + so;
    g.sx[q] = f.sx[q] + so;
    g.sz[q] = f.sz[q] + so;
    g.fz[q] = f.fz[q] + so;
  }
  return g;
}

// The coefficients as seen by one shot: its PML tables, interface rows,
// Ricker table, receiver rows and source position.
__device__ __forceinline__ Coef shot_coef(const Coef& C, int shot) {
  Coef c = C;
  if (shot > 0) {
    const size_t so = size_t(shot) * C.shot_stride;
    c.pmlx = reinterpret_cast<const float4*>(reinterpret_cast<const float*>(C.pmlx) + so);
    c.pmlz = reinterpret_cast<const float4*>(reinterpret_cast<const float*>(C.pmlz) + so);
    c.pmlzf = reinterpret_cast<const float4*>(reinterpret_cast<const float*>(C.pmlzf) + so);
    c.ipre = C.ipre + so;
    c.src_amp = C.src_amp + size_t(shot) * C.src_stride;
    if (C.rec) c.rec = C.rec + size_t(shot) * C.rec_stride;
  }
  if (C.src_pos) {
    const int2 p = __ldg(C.src_pos + shot);
    c.srcx = p.x;
    c.srcz = p.y;
  }
  return c;
}

__constant__ float c_srcw[25];  // 5x5 source spreading weights (src/elements.cu:34-40)
__constant__ float c_w7[7];     // interface filter weights (src/elements.cu:30-33)

template <class T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

// Biased derivative from five taps f(-3..+3) around the centre (tools_func.cuh:50-92).
template <int DIR>
__device__ __forceinline__ float d5(float m3, float m2, float m1, float c0, float p1, float p2,
                                    float p3) {
  if (DIR == kDirF) return kAm1 * m1 + kA0 * c0 + kA1 * p1 + kA2 * p2 + kA3 * p3;
  return -kAm1 * p1 - kA0 * c0 - kA1 * m1 - kA2 * m2 - kA3 * m3;
}

// Zeta derivative with the order lowered near a boundary (tools_func.cuh:94-140).
// `col(j)` returns the value j rows away in the same column.
template <int DIR, class Col>
__device__ __forceinline__ float dz_near(const Col& col, int dist, bool solid_side) {
  if (dist >= 3) return d5<DIR>(col(-3), col(-2), col(-1), col(0), col(1), col(2), col(3));
  if (dist == 2) {
    if (DIR == kDirF) return kM42_0 * col(0) + kM42_1 * col(1) + kM42_2 * col(2);
    return -kM42_0 * col(0) - kM42_1 * col(-1) - kM42_2 * col(-2);
  }
  const bool fwd = (dist == 1) ? (DIR == kDirF) : solid_side;
  if (fwd) return -1.0f * col(0) + 1.0f * col(1);
  return 1.0f * col(0) - 1.0f * col(-1);
}

// The biased derivative of a two-component flux (tools_func.cuh:142-188).
template <int DIR, class Fn>
__device__ __forceinline__ float2 dflux(const Fn& F) {
  if (DIR == kDirF) {
    const float2 m1 = F(-1), c0 = F(0), p1 = F(1), p2 = F(2), p3 = F(3);
    return make_float2(kAm1 * m1.x + kA0 * c0.x + kA1 * p1.x + kA2 * p2.x + kA3 * p3.x,
                       kAm1 * m1.y + kA0 * c0.y + kA1 * p1.y + kA2 * p2.y + kA3 * p3.y);
  }
  const float2 p1 = F(1), c0 = F(0), m1 = F(-1), m2 = F(-2), m3 = F(-3);
  return make_float2(-(kAm1 * p1.x + kA0 * c0.x + kA1 * m1.x + kA2 * m2.x + kA3 * m3.x),
                     -(kAm1 * p1.y + kA0 * c0.y + kA1 * m1.y + kA2 * m2.y + kA3 * m3.y));
}

// Slot of column ix in the xi-strip arrays (valid only where the cell is in a side strip).
__device__ __forceinline__ int xstrip_col(int ix, int nx, int npd) {
  return (ix - 3 < npd) ? ix - 3 : npd + ix - (nx - 3 - npd);
}

// The density slots of the coefficient blocks hold 1/rho (FP64 reciprocal
// rounded once) and the momentum RHS multiplies by it instead of dividing
// (reference: `rhodvx_dt / Mf.rho[idx]`, pml_fs_kernels.cuh:432); the two
// differ by at most one rounding. Build with MFDM_RCP_RHO=0 to divide.
#ifndef MFDM_RCP_RHO
#define MFDM_RCP_RHO 1
#endif
__device__ __forceinline__ float over_rho(float x, float r) {
#if MFDM_RCP_RHO
  return x * r;
#else
  return x / r;
#endif
}

// Direct reads of the stage input (the interface strip and the gradient kernels).
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

// Centre-cell coefficients of a fluid / solid cell (metric at the cell's global row).
struct FluidCoefs { float xix, xiz, zex, zez, rho, K; };
struct SolidCoefs { float xix, xiz, zex, zez, rho, c11, c13, c33, c55; };

__device__ __forceinline__ FluidCoefs fluid_coefs_global(const Coef& C, size_t g) {
  return {ldg(C.xix + g), ldg(C.xiz + g), ldg(C.zex + g), ldg(C.zez + g), ldg(C.rhof + g),
          ldg(C.K + g)};
}
__device__ __forceinline__ SolidCoefs solid_coefs_global(const Coef& C, size_t m, size_t g) {
  return {ldg(C.xix + g), ldg(C.xiz + g), ldg(C.zex + g), ldg(C.zez + g), ldg(C.rhos + m),
          ldg(C.C11 + m), ldg(C.C13 + m), ldg(C.C33 + m), ldg(C.C55 + m)};
}

// Output of the right-hand side at one fluid cell.
struct FluidK {
  float vx, vz, p;
  float V0, V1, E0, E1;      // xi-ADE RHS (valid only in the side strips)
  float ZV0, ZV1, ZE0, ZE1;  // zeta-ADE RHS (top band, four-side CPML only)
  bool has_E;                // false on the free-surface row (p fixed)
};

// Output of the right-hand side at one solid cell.
struct SolidK {
  float vx, vz, sx, sz, sxz;
  float XV0, XV1, XE0, XE1;  // xi-ADE RHS (side strips)
  float ZV0, ZV1, ZE0, ZE1;  // zeta-ADE RHS (bottom strip)
};

// Fluid RHS at (iz, ix), iz in [3, nz_f-1] (pml_fs_kernels.cuh:333-507).
// `A` reads the stage input: A.fp(dz, dx), A.fvx(dz, dx), A.fvz(dz, dx) relative
// to the cell; `ade` holds the stage-input ADE memory (V0, V1, E0, E1) of the cell.
// INTERIOR = true: the caller guarantees 6 <= iz <= nz_f-4 (no conservative
// rows, full-order zeta stencils), so those branches compile away.
// With CPML (CFS-PML on all four sides, cpml_kernels.cuh:240-415) the top is
// not a free surface: only the interface rows take the conservative form,
// row 3 is an ordinary row, and `top` cells (rows 3..npd+2) carry a zeta PML
// whose stage-input ADE memory is `zade`.
template <int DIR, bool INTERIOR = false, bool CPML = false, class Acc>
__device__ __forceinline__ FluidK fluid_rhs(const Coef& C, const Acc& A, int iz, int ix,
                                            bool side, const float* ade, const FluidCoefs& cf,
                                            bool top = false, const float* zade = nullptr) {
  FluidK o;
  const int P = C.P, nzf = C.nzf;
  const bool cpml = !INTERIOR && CPML;
  const size_t g = (size_t)iz * P + ix;
  const float xix = cf.xix, xiz = cf.xiz, zex = cf.zex, zez = cf.zez;
  const float gxx = xix * xix + xiz * xiz;
  const int d_if = nzf - 1 - iz, d_fs = cpml ? 3 : iz - 3;
  float4 pml = make_float4(0.f, 0.f, 0.f, 0.f), pmz = pml;
  if (side) pml = ldg(C.pmlx + ix);
  if (top) pmz = ldg(C.pmlzf + iz);

  // ---- momentum: rho dv/dt = -grad p ----
  {
    float rvx, rvz, divx = 0.f, divz = 0.f, divzx = 0.f, divzz = 0.f;
    if (!INTERIOR && (d_if < 3 || d_fs < 3)) {
      // conservative flux form with mirrored ghosts (pml_fs_kernels.cuh:356-415)
      auto Ff = [&](int r) -> float2 {
        const size_t k = (size_t)r * P + ix;
        const float Jk = ldg(C.J + k), pk = A.fp(r - iz, 0);
        return make_float2(-Jk * ldg(C.zex + k) * pk, -Jk * ldg(C.zez + k) * pk);
      };
      auto Fxi = [&](int j) -> float2 {
        const size_t k = g + j;
        const float Jk = ldg(C.J + k), pk = A.fp(0, j);
        return make_float2(-Jk * ldg(C.xix + k) * pk, -Jk * ldg(C.xiz + k) * pk);
      };
      auto Fze = [&](int j) -> float2 {
        const int r = iz + j;
        if (d_if < 3) {
          if (r <= nzf - 1) return Ff(r);
          const float2 a = Ff(nzf - 1), b = Ff(2 * (nzf - 1) - r);  // G = 2F0 - Fn
          return make_float2(2 * a.x - b.x, 2 * a.y - b.y);
        }
        if (r >= 3) return Ff(r);
        const float2 b = Ff(6 - r);  // free-surface image: G = -Fn
        return make_float2(-b.x, -b.y);
      };
      const float2 a = dflux<DIR>(Fxi), b = dflux<DIR>(Fze);
      const float Sx = a.x + b.x, Sz = a.y + b.y, Jc = ldg(C.J + g);
      rvx = Sx / Jc;
      rvz = Sz / Jc;
      if (side) {
        divx = xix * (xix * Sx + xiz * Sz) / (gxx * Jc);
        divz = xiz * (xix * Sx + xiz * Sz) / (gxx * Jc);
      }
      if (top) {
        const float gzz = zex * zex + zez * zez;
        divzx = zex * (zex * Sx + zez * Sz) / (gzz * Jc);
        divzz = zez * (zex * Sx + zez * Sz) / (gzz * Jc);
      }
    } else {
      const float dpdx = d5<DIR>(A.fp(0, -3), A.fp(0, -2), A.fp(0, -1), A.fp(0, 0), A.fp(0, 1),
                                 A.fp(0, 2), A.fp(0, 3));
      const float dpdz = d5<DIR>(A.fp(-3, 0), A.fp(-2, 0), A.fp(-1, 0), A.fp(0, 0), A.fp(1, 0),
                                 A.fp(2, 0), A.fp(3, 0));
      rvx = -(xix * dpdx + zex * dpdz);
      rvz = -(xiz * dpdx + zez * dpdz);
      if (side) {
        const float gxz = xix * zex + xiz * zez;
        divx = -xix * (gxx * dpdx + gxz * dpdz) / gxx;
        divz = -xiz * (gxx * dpdx + gxz * dpdz) / gxx;
      }
      if (top) {
        const float gxz = xix * zex + xiz * zez, gzz = zex * zex + zez * zez;
        divzx = -zex * (gxz * dpdx + gzz * dpdz) / gzz;
        divzz = -zez * (gxz * dpdx + gzz * dpdz) / gzz;
      }
    }
    const float rho = cf.rho;
    o.vx = over_rho(rvx, rho);
    o.vz = over_rho(rvz, rho);
    if (side) {
      const float dpb = pml.x, apdpb = pml.y, invb = pml.z;
      o.V0 = -apdpb * ade[0] + dpb * divx;
      o.V1 = -apdpb * ade[1] + dpb * divz;
      o.vx += over_rho((invb - 1.0f) * divx - invb * ade[0], rho);
      o.vz += over_rho((invb - 1.0f) * divz - invb * ade[1], rho);
    }
    if (top) {
      const float dpb = pmz.x, apdpb = pmz.y, invb = pmz.z;
      o.ZV0 = -apdpb * zade[0] + dpb * divzx;
      o.ZV1 = -apdpb * zade[1] + dpb * divzz;
      o.vx += over_rho((invb - 1.0f) * divzx - invb * zade[0], rho);
      o.vz += over_rho((invb - 1.0f) * divzz - invb * zade[1], rho);
    }
  }
  // ---- pressure: dp/dt = -K div v ----
  o.has_E = INTERIOR || cpml || (iz != 3);
  if (!INTERIOR && !cpml && iz == 3) {
    o.p = 0.0f;  // pressure-free surface row
  } else {
    auto vxc = [&](int j) { return A.fvx(j, 0); };
    auto vzc = [&](int j) { return A.fvz(j, 0); };
    const float dvxdx = d5<DIR>(A.fvx(0, -3), A.fvx(0, -2), A.fvx(0, -1), A.fvx(0, 0),
                                A.fvx(0, 1), A.fvx(0, 2), A.fvx(0, 3));
    const float dvzdx = d5<DIR>(A.fvz(0, -3), A.fvz(0, -2), A.fvz(0, -1), A.fvz(0, 0),
                                A.fvz(0, 1), A.fvz(0, 2), A.fvz(0, 3));
    const int dn = INTERIOR ? 3 : (cpml ? nzf - 1 - iz : min(iz - 3, nzf - 1 - iz));
    const float dvxdz = dz_near<DIR>(vxc, dn, false);
    const float dvzdz = dz_near<DIR>(vzc, dn, false);
    const float Kc = cf.K;
    o.p = -Kc * (xix * dvxdx + zex * dvxdz + xiz * dvzdx + zez * dvzdz);
    if (side) {
      const float gxz = xix * zex + xiz * zez;
      const float Dvx = dvxdx + (gxz / gxx) * dvxdz, Dvz = dvzdx + (gxz / gxx) * dvzdz;
      const float dpb = pml.x, apdpb = pml.y, invb = pml.z;
      o.E0 = -apdpb * ade[2] + dpb * Dvx;
      o.E1 = -apdpb * ade[3] + dpb * Dvz;
      if (CPML)  // the four-side variant multiplies K into each term (cpml_kernels.cuh:390-395)
        o.p += -Kc * (invb - 1.0f) * xix * Dvx - Kc * (invb - 1.0f) * xiz * Dvz +
               invb * Kc * xix * ade[2] + invb * Kc * xiz * ade[3];
      else
        o.p += Kc * (-(invb - 1.0f) * xix * Dvx - (invb - 1.0f) * xiz * Dvz +
                     invb * xix * ade[2] + invb * xiz * ade[3]);
    }
    if (top) {
      const float gxz = xix * zex + xiz * zez, gzz = zex * zex + zez * zez;
      const float Dzx = dvxdz + (gxz / gzz) * dvxdx, Dzz = dvzdz + (gxz / gzz) * dvzdx;
      const float dpb = pmz.x, apdpb = pmz.y, invb = pmz.z;
      o.ZE0 = -apdpb * zade[2] + dpb * Dzx;
      o.ZE1 = -apdpb * zade[3] + dpb * Dzz;
      o.p += Kc * (-(invb - 1.0f) * (zex * Dzx + zez * Dzz) + invb * (zex * zade[2] + zez * zade[3]));
    }
  }
  return o;
}

// Solid RHS at (iz, ix), iz in [0, nz_s-4] (pml_fs_kernels.cuh:509-752).
// `A` reads the stage input: A.svx, A.svz, A.ssx, A.ssz, A.ssxz (dz, dx);
// `xade` / `zade` are the stage-input xi / zeta ADE memory of the cell.
// INTERIOR = true: the caller guarantees 3 <= iz <= nz_s-4.
template <int DIR, bool INTERIOR = false, bool CPML = false, class Acc>
__device__ __forceinline__ SolidK solid_rhs(const Coef& C, const Acc& A, int iz, int ix, bool side,
                                            bool bottom, const float* xade, const float* zade,
                                            const SolidCoefs& cf) {
  SolidK o;
  const int P = C.P, nzf = C.nzf;
  const size_t m = (size_t)iz * P + ix;
  const size_t g = m + (size_t)(nzf - 1) * P;
  const float xix = cf.xix, xiz = cf.xiz, zex = cf.zex, zez = cf.zez;
  float4 px = make_float4(0.f, 0.f, 0.f, 0.f), pz = px;
  if (side) px = ldg(C.pmlx + ix);
  if (bottom) pz = ldg(C.pmlz + iz);

  // ---- momentum: rho dv/dt = div sigma ----
  {
    float rvx, rvz, dxx = 0.f, dxz = 0.f, dzx = 0.f, dzz = 0.f;
    if (!INTERIOR && iz < 3) {
      // conservative flux form with the interface ghost G = 2F0 - Fn (pml_fs_kernels.cuh:654-680)
      auto Fs = [&](int r) -> float2 {
        const size_t k = (size_t)(r + nzf - 1) * P + ix;
        const float Jk = ldg(C.J + k), ax = ldg(C.zex + k), az = ldg(C.zez + k);
        const int dz = r - iz;
        return make_float2(Jk * (ax * A.ssx(dz, 0) + az * A.ssxz(dz, 0)),
                           Jk * (ax * A.ssxz(dz, 0) + az * A.ssz(dz, 0)));
      };
      auto Fxi = [&](int j) -> float2 {
        const size_t k = g + j;
        const float Jk = ldg(C.J + k), ax = ldg(C.xix + k), az = ldg(C.xiz + k);
        return make_float2(Jk * (ax * A.ssx(0, j) + az * A.ssxz(0, j)),
                           Jk * (ax * A.ssxz(0, j) + az * A.ssz(0, j)));
      };
      auto Fze = [&](int j) -> float2 {
        const int r = iz + j;
        if (r >= 0) return Fs(r);
        const float2 a = Fs(0), b = Fs(-r);
        return make_float2(2 * a.x - b.x, 2 * a.y - b.y);
      };
      const float2 a = dflux<DIR>(Fxi), b = dflux<DIR>(Fze);
      const float Sx = a.x + b.x, Sz = a.y + b.y, Jc = ldg(C.J + g);
      rvx = Sx / Jc;
      rvz = Sz / Jc;
      if (side) {
        const float gxx = xix * xix + xiz * xiz;
        dxx = xix * (xix * Sx + xiz * Sz) / (gxx * Jc);
        dxz = xiz * (xix * Sx + xiz * Sz) / (gxx * Jc);
      }
      if (bottom) {
        const float gzz = zex * zex + zez * zez;
        dzx = zex * (zex * Sx + zez * Sz) / (gzz * Jc);
        dzz = zez * (zex * Sx + zez * Sz) / (gzz * Jc);
      }
    } else {
      const float sxdx = d5<DIR>(A.ssx(0, -3), A.ssx(0, -2), A.ssx(0, -1), A.ssx(0, 0),
                                 A.ssx(0, 1), A.ssx(0, 2), A.ssx(0, 3));
      const float sxdz = d5<DIR>(A.ssx(-3, 0), A.ssx(-2, 0), A.ssx(-1, 0), A.ssx(0, 0),
                                 A.ssx(1, 0), A.ssx(2, 0), A.ssx(3, 0));
      const float szdx = d5<DIR>(A.ssz(0, -3), A.ssz(0, -2), A.ssz(0, -1), A.ssz(0, 0),
                                 A.ssz(0, 1), A.ssz(0, 2), A.ssz(0, 3));
      const float szdz = d5<DIR>(A.ssz(-3, 0), A.ssz(-2, 0), A.ssz(-1, 0), A.ssz(0, 0),
                                 A.ssz(1, 0), A.ssz(2, 0), A.ssz(3, 0));
      const float tdx = d5<DIR>(A.ssxz(0, -3), A.ssxz(0, -2), A.ssxz(0, -1), A.ssxz(0, 0),
                                A.ssxz(0, 1), A.ssxz(0, 2), A.ssxz(0, 3));
      const float tdz = d5<DIR>(A.ssxz(-3, 0), A.ssxz(-2, 0), A.ssxz(-1, 0), A.ssxz(0, 0),
                                A.ssxz(1, 0), A.ssxz(2, 0), A.ssxz(3, 0));
      rvx = xix * sxdx + zex * sxdz + xiz * tdx + zez * tdz;
      rvz = xix * tdx + zex * tdz + xiz * szdx + zez * szdz;
      if (side || bottom) {
        const float gxz = xix * zex + xiz * zez;
        if (side) {
          const float gxx = xix * xix + xiz * xiz;
          dxx = xix * (sxdx + gxz / gxx * sxdz) + xiz * (tdx + gxz / gxx * tdz);
          dxz = xix * (tdx + gxz / gxx * tdz) + xiz * (szdx + gxz / gxx * szdz);
        }
        if (bottom) {
          const float gzz = zex * zex + zez * zez;
          dzx = zex * (sxdz + gxz / gzz * sxdx) + zez * (gxz / gzz * tdx + tdz);
          dzz = zex * (gxz / gzz * tdx + tdz) + zez * (gxz / gzz * szdx + szdz);
        }
      }
    }
    const float rho = cf.rho;
    o.vx = over_rho(rvx, rho);
    o.vz = over_rho(rvz, rho);
    if (side) {
      const float dpb = px.x, apdpb = px.y, invb = px.z;
      o.XV0 = -apdpb * xade[0] + dpb * dxx;
      o.XV1 = -apdpb * xade[1] + dpb * dxz;
      o.vx += over_rho((invb - 1.0f) * dxx - invb * xade[0], rho);
      o.vz += over_rho((invb - 1.0f) * dxz - invb * xade[1], rho);
    }
    if (bottom) {
      const float dpb = pz.x, apdpb = pz.y, invb = pz.z;
      o.ZV0 = -apdpb * zade[0] + dpb * dzx;
      o.ZV1 = -apdpb * zade[1] + dpb * dzz;
      o.vx += over_rho((invb - 1.0f) * dzx - invb * zade[0], rho);
      o.vz += over_rho((invb - 1.0f) * dzz - invb * zade[1], rho);
    }
  }
  // ---- stress: VTI constitutive law ----
  {
    auto vxc = [&](int j) { return A.svx(j, 0); };
    auto vzc = [&](int j) { return A.svz(j, 0); };
    const float dvxdx = d5<DIR>(A.svx(0, -3), A.svx(0, -2), A.svx(0, -1), A.svx(0, 0),
                                A.svx(0, 1), A.svx(0, 2), A.svx(0, 3));
    const float dvzdx = d5<DIR>(A.svz(0, -3), A.svz(0, -2), A.svz(0, -1), A.svz(0, 0),
                                A.svz(0, 1), A.svz(0, 2), A.svz(0, 3));
    const float dvxdz = dz_near<DIR>(vxc, INTERIOR ? 3 : iz, true);
    const float dvzdz = dz_near<DIR>(vzc, INTERIOR ? 3 : iz, true);
    const float c11 = cf.c11, c13 = cf.c13, c33 = cf.c33, c55 = cf.c55;
    o.sx = c11 * (xix * dvxdx + zex * dvxdz) + c13 * (xiz * dvzdx + zez * dvzdz);
    o.sz = c13 * (xix * dvxdx + zex * dvxdz) + c33 * (xiz * dvzdx + zez * dvzdz);
    if (CPML) {
      // The four-side variant reads this line's metric with the solid-local
      // index, i.e. at global row iz (cpml_kernels.cuh:448-455); kept for parity.
      const size_t b = (size_t)iz * C.P + ix;
      o.sxz = c55 * (ldg(C.xiz + b) * dvxdx + ldg(C.zez + b) * dvxdz + ldg(C.xix + b) * dvzdx +
                     ldg(C.zex + b) * dvzdz);
    } else {
      o.sxz = c55 * (xiz * dvxdx + zez * dvxdz + xix * dvzdx + zex * dvzdz);
    }
    if (side || bottom) {
      const float gxz = xix * zex + xiz * zez;
      if (side) {
        const float gxx = xix * xix + xiz * xiz;
        const float Dvx = dvxdx + (gxz / gxx) * dvxdz, Dvz = dvzdx + (gxz / gxx) * dvzdz;
        const float dpb = px.x, apdpb = px.y, invb = px.z;
        const float E0 = xade[2], E1 = xade[3];
        o.XE0 = -apdpb * E0 + dpb * Dvx;
        o.XE1 = -apdpb * E1 + dpb * Dvz;
        o.sx += c11 * (invb - 1.0f) * xix * Dvx + c13 * (invb - 1.0f) * xiz * Dvz -
                invb * c11 * xix * E0 - invb * c13 * xiz * E1;
        o.sz += c13 * (invb - 1.0f) * xix * Dvx + c33 * (invb - 1.0f) * xiz * Dvz -
                invb * c13 * xix * E0 - invb * c33 * xiz * E1;
        o.sxz += c55 * (invb - 1.0f) * (xiz * Dvx + xix * Dvz) - invb * c55 * xiz * E0 -
                 invb * c55 * xix * E1;
      }
      if (bottom) {
        const float gzz = zex * zex + zez * zez;
        const float Dvx = dvxdz + (gxz / gzz) * dvxdx, Dvz = dvzdz + (gxz / gzz) * dvzdx;
        const float dpb = pz.x, apdpb = pz.y, invb = pz.z;
        const float E0 = zade[2], E1 = zade[3];
        o.ZE0 = -apdpb * E0 + dpb * Dvx;
        o.ZE1 = -apdpb * E1 + dpb * Dvz;
        o.sx += c11 * (invb - 1.0f) * zex * Dvx + c13 * (invb - 1.0f) * zez * Dvz -
                invb * c11 * zex * E0 - invb * c13 * zez * E1;
        o.sz += c13 * (invb - 1.0f) * zex * Dvx + c33 * (invb - 1.0f) * zez * Dvz -
                invb * c13 * zex * E0 - invb * c33 * zez * E1;
        o.sxz += c55 * (invb - 1.0f) * (zez * Dvx + zex * Dvz) - invb * c55 * zez * E0 -
                 invb * c55 * zex * E1;
      }
    }
  }
  return o;
}

// Normal/tangential coupling of the stage RHS on the interface
// (pml_fs_kernels.cuh:754-827): kf = fluid (vx, vz, p), ks = solid (vx, vz,
// sx, sz, sxz) RHS of one column, kv = the eight coupled values in that order.
// Direction F: the fluid takes the solid's normal velocity and traction;
// B: the solid takes the fluid's.
template <int DIR>
__device__ __forceinline__ void couple_rhs(float2 n, const float* kf, const float* ks, float* kv) {
  const float vxf = kf[0], vzf = kf[1];
  float pf = kf[2];
  const float vxs = ks[0], vzs = ks[1], sxx = ks[2], szz = ks[3], sxz = ks[4];
  float vnf = n.x * vxf + n.y * vzf;
  const float vtf = n.y * vxf - n.x * vzf;
  float vns = n.x * vxs + n.y * vzs;
  const float vts = n.y * vxs - n.x * vzs;
  float snn = n.x * n.x * sxx + 2 * n.x * n.y * sxz + n.y * n.y * szz;
  float snt = n.x * n.y * (sxx - szz) + (n.y * n.y - n.x * n.x) * sxz;
  const float stt = n.y * n.y * sxx - 2 * n.x * n.y * sxz + n.x * n.x * szz;
  if (DIR == kDirF) {
    vnf = vns;
    pf = -snn;
    snt = 0.f;
  } else {
    vns = vnf;
    snn = -pf;
    snt = 0.f;
  }
  kv[0] = n.x * vnf + n.y * vtf;
  kv[1] = n.y * vnf - n.x * vtf;
  kv[2] = pf;
  kv[3] = n.x * vns + n.y * vts;
  kv[4] = n.y * vns - n.x * vts;
  kv[5] = n.x * n.x * snn + 2 * n.x * n.y * snt + n.y * n.y * stt;
  kv[6] = n.y * n.y * snn - 2 * n.x * n.y * snt + n.x * n.x * stt;
  kv[7] = -n.x * n.y * stt + (n.y * n.y - n.x * n.x) * snt;
}

// Continuity average of the filtered interface values (src/pml_fs_kernels.cu:
// 470-520): v = filtered (fluid vx, vz, p, solid vx, vz, sx, sz, sxz) of one
// column, u = the new interface state in the same order.
__device__ __forceinline__ void interface_average(float2 n, const float* v, float* u) {
  const float vnf = n.x * v[0] + n.y * v[1], vtf = n.y * v[0] - n.x * v[1];
  const float vns = n.x * v[3] + n.y * v[4], vts = n.y * v[3] - n.x * v[4];
  const float snn = n.x * n.x * v[5] + 2.0f * n.x * n.y * v[7] + n.y * n.y * v[6];
  const float stt = n.y * n.y * v[5] - 2.0f * n.x * n.y * v[7] + n.x * n.x * v[6];
  const float vn = 0.5f * (vnf + vns);
  const float sn = 0.5f * (snn - v[2]);
  u[0] = n.x * vn + n.y * vtf;
  u[1] = n.y * vn - n.x * vtf;
  u[2] = -sn;
  u[3] = n.x * vn + n.y * vts;
  u[4] = n.y * vn - n.x * vts;
  u[5] = n.x * n.x * sn + n.y * n.y * stt;
  u[6] = n.y * n.y * sn + n.x * n.x * stt;
  u[7] = n.x * n.y * (sn - stt);
}

// Source term of stage `s` at fluid cell (iz, ix): 5x5 Gaussian spreading of the
// Ricker value, skipped within 3 cells of any edge (tools_func.cuh:21-37).
__device__ __forceinline__ float source_term(const Coef& C, int iz, int ix, int it, int s) {
  const int dx = ix - C.srcx, dz = iz - C.srcz;
  if (C.srcx < 0 || dx < -2 || dx > 2 || dz < -2 || dz > 2) return 0.0f;
  if (ix <= 2 || ix >= C.nx - 3 || iz <= 2 || iz >= C.nzf - 3) return 0.0f;
  const int row = it - C.src_it0;
  if (row < 0 || row >= C.src_steps) return 0.0f;
  const float amp = ldg(C.src_amp + (size_t)row * 4 + s);
  return amp * c_srcw[(dz + 2) * 5 + (dx + 2)];
}

// RK4 bookkeeping for one value (src/pml_fs_kernels.cu:663-763, fused):
//   first stage: out = u + c k,  acc = u + w k
//   middle:      out = Un + c k, acc += w k
//   last:        out = acc + c k
template <int KIND>
__device__ __forceinline__ void rk_update(float k, float uin, const float* __restrict__ Un,
                                          float* __restrict__ out, float* __restrict__ acc,
                                          size_t i, float c, float w) {
  if (KIND == kStageFirst) {
    out[i] = fmaf(c, k, uin);
    acc[i] = fmaf(w, k, uin);
  } else if (KIND == kStageMid) {
    out[i] = fmaf(c, k, Un[i]);
    acc[i] = fmaf(w, k, acc[i]);
  } else {
    out[i] = fmaf(c, k, acc[i]);
  }
}

}  // namespace mfdm
