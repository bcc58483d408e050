// sm_100a kernels of the solid-only time step with a free surface (see mfdm_solid.h).
//
// One launch per RK stage does the whole stage: velocity and stress
// right-hand sides of every cell (the reference's update_velocity and
// update_stress, which run as two kernels on two streams), the free-surface
// ghost fluxes (built on the fly from the stage input instead of a separate
// build_ghost_flux launch), the explosive source and the fused RK4 update
// (the reference's vector_add / vector_self_add launches over full grids).
// A fifth launch per step samples the receiver row and advances the device
// step counter. Reads go through the read-only cache: at the sizes of
// solid-only runs a cell's 5x5 neighbourhood is served from L1/L2.
#include "mfdm_device.cuh"
#include "mfdm_solid.h"

namespace mfdm {
namespace solid {
namespace {

constexpr int kBX = 32, kBY = 8;

struct SrcW { float w[25]; };

struct Out {
  float vx, vz, sx, sz, sxz;
  float XV0, XV1, XE0, XE1, ZV0, ZV1, ZE0, ZE1;
};

// Right-hand side of cell (iz, ix), 3 <= iz <= nz-4 (include/pml_fs_kernels.cuh:10-307).
template <int DIR>
__device__ __forceinline__ Out rhs(const SCoef& C, const SFields& S, int iz, int ix) {
  Out o;
  const int P = C.P, nx = C.nx, nz = C.nz, npd = C.npd;
  const size_t i = (size_t)iz * P + ix;
  const int dist = iz - 3, distx = min(ix - 3, nx - 4 - ix);
  const bool side = distx < npd, bottom = iz >= nz - 3 - npd;
  const int scol = side ? xstrip_col(ix, nx, npd) : 0;
  const size_t si = (size_t)iz * C.Ps + scol, zi = (size_t)(iz - (nz - 3 - npd)) * P + ix;
  const float xix = __ldg(C.xix + i), xiz = __ldg(C.xiz + i), zex = __ldg(C.zex + i),
              zez = __ldg(C.zez + i);
  const float gxixi = xix * xix + xiz * xiz, gzeze = zex * zex + zez * zez;
  const float gxize = xix * zex + xiz * zez;
  auto at = [&](const float* f, int dz, int dx) { return __ldg(f + i + (ptrdiff_t)dz * P + dx); };
  auto dx5 = [&](const float* f) {
    return d5<DIR>(at(f, 0, -3), at(f, 0, -2), at(f, 0, -1), at(f, 0, 0), at(f, 0, 1), at(f, 0, 2),
                   at(f, 0, 3));
  };
  auto dzn = [&](const float* f, int d) {
    auto col = [&](int j) { return at(f, j, 0); };
    return dz_near<DIR>(col, d, true);
  };
  o.XV0 = o.XV1 = o.XE0 = o.XE1 = o.ZV0 = o.ZV1 = o.ZE0 = o.ZE1 = 0.f;

  // ---- momentum: rho dv/dt = div sigma ----
  {
    float rvx, rvz, dxx, dxz, dzx = 0.f, dzz = 0.f;
    if (dist < 3) {
      // conservative rows under the free surface; above it the image G = -F of
      // the rows below (src/pml_fs_kernels.cu:7-19)
      auto Fs = [&](int r) -> float2 {
        const size_t k = (size_t)r * P + ix;
        const float Jk = __ldg(C.J + k), ax = __ldg(C.zex + k), az = __ldg(C.zez + k);
        const float sx = __ldg(S.sx + k), sz = __ldg(S.sz + k), sxz = __ldg(S.sxz + k);
        return make_float2(Jk * (ax * sx + az * sxz), Jk * (ax * sxz + az * sz));
      };
      auto Fxi = [&](int j) -> float2 {
        const size_t k = i + j;
        const float Jk = __ldg(C.J + k), ax = __ldg(C.xix + k), az = __ldg(C.xiz + k);
        const float sx = __ldg(S.sx + k), sz = __ldg(S.sz + k), sxz = __ldg(S.sxz + k);
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
      const float dxsx = dx5(S.sx), dxsz = dx5(S.sz), dxsxz = dx5(S.sxz);
      const float dzsx = dzn(S.sx, dist), dzsz = dzn(S.sz, dist), dzsxz = dzn(S.sxz, dist);
      dxx = xix * (dxsx + gxize / gxixi * dzsx) + xiz * (dxsxz + gxize / gxixi * dzsxz);
      dxz = xix * (dxsxz + gxize / gxixi * dzsxz) + xiz * (dxsz + gxize / gxixi * dzsz);
    } else {
      const float sxdx = dx5(S.sx), sxdz = dzn(S.sx, 3), szdx = dx5(S.sz), szdz = dzn(S.sz, 3);
      const float tdx = dx5(S.sxz), tdz = dzn(S.sxz, 3);
      rvx = xix * sxdx + zex * sxdz + xiz * tdx + zez * tdz;
      rvz = xix * tdx + zex * tdz + xiz * szdx + zez * szdz;
      dxx = xix * (sxdx + gxize / gxixi * sxdz) + xiz * (tdx + gxize / gxixi * tdz);
      dxz = xix * (tdx + gxize / gxixi * tdz) + xiz * (szdx + gxize / gxixi * szdz);
      dzx = zex * (sxdz + gxize / gzeze * sxdx) + zez * (gxize / gzeze * tdx + tdz);
      dzz = zex * (gxize / gzeze * tdx + tdz) + zez * (gxize / gzeze * szdx + szdz);
    }
    const float r0 = __ldg(C.rho + i);
    o.vx = rvx / r0;
    o.vz = rvz / r0;
    if (side) {
      const float4 p = __ldg(C.pmlx + ix);
      const float V0 = __ldg(S.x[0] + si), V1 = __ldg(S.x[1] + si);
      o.XV0 = -p.y * V0 + p.x * dxx;
      o.XV1 = -p.y * V1 + p.x * dxz;
      o.vx += ((p.z - 1.0f) * dxx - p.z * V0) / r0;
      o.vz += ((p.z - 1.0f) * dxz - p.z * V1) / r0;
    }
    if (bottom) {
      const float4 p = __ldg(C.pmlz + iz);
      const float V0 = __ldg(S.z[0] + zi), V1 = __ldg(S.z[1] + zi);
      o.ZV0 = -p.y * V0 + p.x * dzx;
      o.ZV1 = -p.y * V1 + p.x * dzz;
      o.vx += ((p.z - 1.0f) * dzx - p.z * V0) / r0;
      o.vz += ((p.z - 1.0f) * dzz - p.z * V1) / r0;
    }
  }
  // ---- stress ----
  {
    const float c11 = __ldg(C.C11 + i), c13 = __ldg(C.C13 + i), c33 = __ldg(C.C33 + i),
                c55 = __ldg(C.C55 + i);
    const float dvx_dxi = dx5(S.vx), dvz_dxi = dx5(S.vz);
    if (dist == 0) {
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
    const float dvx_dze = dzn(S.vx, dist), dvz_dze = dzn(S.vz, dist);
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

template <int DIR, int KIND>
__global__ void __launch_bounds__(kBX * kBY) k_stage(SCoef C, SFields in, SFields out, SFields un,
                                                      SFields acc, int s, float c, float w, SrcW W) {
  const int ix = 3 + blockIdx.x * kBX + threadIdx.x, iz = 3 + blockIdx.y * kBY + threadIdx.y;
  const int nx = C.nx, nz = C.nz, npd = C.npd, P = C.P;
  if (ix > nx - 4 || iz > nz - 4) return;
  Out o = rhs<DIR>(C, in, iz, ix);
  // explosive source on both normal stresses (src/pml_fs_kernels.cu:22-26)
  const int it = __ldg(C.step);
  const int sx = ix - C.srcx, sz = iz - C.srcz;
  if (C.srcx >= 0 && sx >= -2 && sx <= 2 && sz >= -2 && sz <= 2 && it >= 0 && it < C.src_steps) {
    const float q = __ldg(C.src_amp + (size_t)it * 4 + s) * W.w[(sz + 2) * 5 + (sx + 2)];
    o.sx += q;
    o.sz += q;
  }
  const size_t i = (size_t)iz * P + ix;
  upd<KIND>(o.vx, in.vx, un.vx, out.vx, acc.vx, i, c, w);
  upd<KIND>(o.vz, in.vz, un.vz, out.vz, acc.vz, i, c, w);
  upd<KIND>(o.sx, in.sx, un.sx, out.sx, acc.sx, i, c, w);
  upd<KIND>(o.sz, in.sz, un.sz, out.sz, acc.sz, i, c, w);
  upd<KIND>(o.sxz, in.sxz, un.sxz, out.sxz, acc.sxz, i, c, w);
  if (min(ix - 3, nx - 4 - ix) < npd) {
    const size_t si = (size_t)iz * C.Ps + xstrip_col(ix, nx, npd);
    upd<KIND>(o.XV0, in.x[0], un.x[0], out.x[0], acc.x[0], si, c, w);
    upd<KIND>(o.XV1, in.x[1], un.x[1], out.x[1], acc.x[1], si, c, w);
    upd<KIND>(o.XE0, in.x[2], un.x[2], out.x[2], acc.x[2], si, c, w);
    upd<KIND>(o.XE1, in.x[3], un.x[3], out.x[3], acc.x[3], si, c, w);
  }
  if (iz >= nz - 3 - npd) {
    const size_t zi = (size_t)(iz - (nz - 3 - npd)) * P + ix;
    upd<KIND>(o.ZV0, in.z[0], un.z[0], out.z[0], acc.z[0], zi, c, w);
    upd<KIND>(o.ZV1, in.z[1], un.z[1], out.z[1], acc.z[1], zi, c, w);
    upd<KIND>(o.ZE0, in.z[2], un.z[2], out.z[2], acc.z[2], zi, c, w);
    upd<KIND>(o.ZE1, in.z[3], un.z[3], out.z[3], acc.z[3], zi, c, w);
  }
}

__global__ void k_finish(SCoef C, SFields U) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int it = *C.step;
  if (ix < C.nx) {
    const float v = U.vz[(size_t)3 * C.P + ix];
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
  // the 5x5 source weights (src/elements.cu:34-40)
  const SrcW W{{0.0030f, 0.0133f, 0.0219f, 0.0133f, 0.0030f, 0.0133f, 0.0596f, 0.0983f, 0.0596f,
                0.0133f, 0.0219f, 0.0983f, 0.1621f, 0.0983f, 0.0219f, 0.0133f, 0.0596f, 0.0983f,
                0.0596f, 0.0133f, 0.0030f, 0.0133f, 0.0219f, 0.0133f, 0.0030f}};
  const dim3 grid(unsigned((C.nx - 6 + kBX - 1) / kBX), unsigned((C.nz - 6 + kBY - 1) / kBY));
  const float c = C.rk_c[s], w = KIND == kStageLast ? 0.f : C.rk_w[s];
  k_stage<DIR, KIND><<<grid, dim3(kBX, kBY), 0, st>>>(C, in, out, un, acc, s, c, w, W);
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
