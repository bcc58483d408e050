// sm_100a kernels of the adjoint-state backward (see mfdm_adjoint.h).
#include <cub/device/device_scan.cuh>

#include <algorithm>

#include "mfdm_adjoint.h"

namespace mfdm {
namespace adj {
namespace {

#ifndef MFDM_CSR_LANES
#define MFDM_CSR_LANES 2
#endif
constexpr int kLanes = MFDM_CSR_LANES;  // threads per CSR row in the transposed products
static_assert(kLanes == 1 || kLanes == 2 || kLanes == 4 || kLanes == 8 || kLanes == 16, "lanes per CSR row");
constexpr int kBlock = 256;

__device__ __forceinline__ int strip_to_col(int s, int nx, int npd) {
  return s < npd ? 3 + s : nx - 3 - npd + (s - npd);
}
__device__ __forceinline__ int col_to_strip(int c, int nx, int npd) {
  if (c >= 3 && c < 3 + npd) return c - 3;
  if (c >= nx - 3 - npd && c < nx - 3) return npd + c - (nx - 3 - npd);
  return -1;
}

// Global (row, column) of cell (r, c) of array a.
__device__ __forceinline__ void to_global(const SetLayout& L, int a, int r, int c, int& gr, int& gc) {
  switch (L.kind[a]) {
    case 0: gr = r; gc = c; break;
    case 1: gr = L.nzf - 1 + r; gc = c; break;
    case 2: gr = r; gc = strip_to_col(c, L.nx, L.npd); break;
    case 3: gr = L.nzf - 1 + r; gc = strip_to_col(c, L.nx, L.npd); break;
    case 4: gr = L.nzf - 1 + (L.nzs - 3 - L.npd) + r; gc = c; break;
    default: gr = 3 + r; gc = c; break;
  }
}

// Cell (r, c) of array a at global (gr, gc); false if a has no such cell.
__device__ __forceinline__ bool to_local(const SetLayout& L, int a, int gr, int gc, int& r, int& c) {
  if (gc < 0 || gc >= L.nx) return false;
  switch (L.kind[a]) {
    case 0: r = gr; c = gc; break;
    case 1: r = gr - (L.nzf - 1); c = gc; break;
    case 2: r = gr; c = col_to_strip(gc, L.nx, L.npd); break;
    case 3: r = gr - (L.nzf - 1); c = col_to_strip(gc, L.nx, L.npd); break;
    case 4: r = gr - (L.nzf - 1) - (L.nzs - 3 - L.npd); c = gc; break;
    default: r = gr - 3; c = gc; break;
  }
  return r >= 0 && r < L.rows[a] && c >= 0 && c < L.ncols[a];
}

// Offset in [-3, 3] from v to the nearest value congruent to t modulo 7.
__device__ __forceinline__ int lattice_offset(int t, int v) {
  int m = (t - v) % 7;
  if (m < 0) m += 7;
  return m > 3 ? m - 7 : m;
}

// Array, row and column of float i of a set; false for padding.
__device__ __forceinline__ bool locate(const SetLayout& L, long long i, int& a, int& r, int& c) {
  a = -1;
#pragma unroll
  for (int k = 0; k < kSetArrays; ++k)
    if (L.rows[k] > 0 && i >= L.off[k]) a = k;
  if (a < 0) return false;
  const long long loc = i - L.off[a];
  r = int(loc / L.pitch[a]);
  c = int(loc % L.pitch[a]);
  return r < L.rows[a] && c < L.ncols[a];
}

// Output cells whose stage right-hand side is (cell coefficients) x (biased
// derivatives at the cell) plus point-wise ADE terms, all of it transposed by
// the Q fields and the point-wise ADE transpose: the interior cells and the
// PML strip cells of the same rows (full-order zeta stencils: fluid rows
// 6..nz_f-4, below the top band with four-side CPML; solid rows 3..nz_s-4,
// the bottom band included), main fields and their ADE memory. The interface
// strip, the conservative and one-sided rows and the four-side CPML's fluid
// top band stay in the CSR part.
__device__ __forceinline__ bool structured_cell(const SetLayout& L, int a, int r, int c) {
  const int flo = L.cpml ? max(6, L.npd + 3) : 6;
  switch (L.kind[a]) {
    case 0: return c >= 3 && c <= L.nx - 4 && r >= flo && r <= L.nzf - 4;
    case 1: return c >= 3 && c <= L.nx - 4 && r >= 3 && r <= L.nzs - 4;
    case 2: return r >= flo && r <= L.nzf - 4;
    case 3: return r >= 3 && r <= L.nzs - 4;
    case 4: {
      const int rs = L.nzs - 3 - L.npd + r;
      return rs >= 3 && rs <= L.nzs - 4;
    }
    default: return false;
  }
}

__global__ void k_set_lattice(float* set, SetLayout L, int a, int cz, int cx, float v) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (c >= L.ncols[a] || r >= L.rows[a]) return;
  int gr, gc;
  to_global(L, a, r, c, gr, gc);
  if (gr % 7 == cz && gc % 7 == cx) set[L.off[a] + (long long)r * L.pitch[a] + c] = v;
}

__global__ void k_fill(float* set, long long n, float v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    set[i] = v;
}

__global__ void k_mask(const float* out, uint8_t* mask, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    mask[i] = out[i] != 0.0f ? 1 : 0;
}

__global__ void k_extract(const float* __restrict__ out, SetLayout L, int a, int cz, int cx,
                          float scale, unsigned long long* count, const long long* rowptr,
                          int* cursor, int* col, float* val, int* err) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < L.len;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = out[i];
    if (v == 0.0f) continue;
    int g, r, c;
    if (!locate(L, i, g, r, c)) {
      atomicAdd(err, 1);
      continue;
    }
    int gr, gc, r2, c2;
    to_global(L, g, r, c, gr, gc);
    if (!to_local(L, a, gr + lattice_offset(cz, gr), gc + lattice_offset(cx, gc), r2, c2)) {
      atomicAdd(err, 1);
      continue;
    }
    const long long j = L.off[a] + (long long)r2 * L.pitch[a] + c2;
    if (!rowptr) {
      atomicAdd(count + j, 1ull);
    } else {
      const long long pos = rowptr[j] + atomicAdd(cursor + j, 1);
      col[pos] = int(i);
      val[pos] = v * scale;
    }
  }
}

__global__ void k_sort_rows(const long long* __restrict__ rowptr, int* col, float* val, long long len) {
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= len) return;
  const long long b = rowptr[j], e = rowptr[j + 1];
  for (long long k = b + 1; k < e; ++k) {
    const int ck = col[k];
    const float vk = val[k];
    long long q = k - 1;
    while (q >= b && col[q] > ck) {
      col[q + 1] = col[q];
      val[q + 1] = val[q];
      --q;
    }
    col[q + 1] = ck;
    val[q + 1] = vk;
  }
}

// Row sums of L^T x by groups of kLanes threads (coalesced along each row).
// Each lane loads four of its entries (and their x) before accumulating them,
// in the same order as one at a time, so four gathers are in flight per lane.
__device__ __forceinline__ float row_dot(const long long* __restrict__ rowptr,
                                         const int* __restrict__ col, const float* __restrict__ val,
                                         const float* __restrict__ x, long long row, int lane) {
  float s = 0.0f;
  const long long e = rowptr[row + 1];
  long long k = rowptr[row] + lane;
  for (; k + 3 * kLanes < e; k += 4 * kLanes) {
    const int c0 = col[k], c1 = col[k + kLanes], c2 = col[k + 2 * kLanes], c3 = col[k + 3 * kLanes];
    const float v0 = val[k], v1 = val[k + kLanes], v2 = val[k + 2 * kLanes], v3 = val[k + 3 * kLanes];
    const float x0 = __ldg(x + c0), x1 = __ldg(x + c1), x2 = __ldg(x + c2), x3 = __ldg(x + c3);
    s = fmaf(v0, x0, s);
    s = fmaf(v1, x1, s);
    s = fmaf(v2, x2, s);
    s = fmaf(v3, x3, s);
  }
  for (; k < e; k += kLanes) s = fmaf(val[k], __ldg(x + col[k]), s);
  const unsigned grp = ((1u << kLanes) - 1u) << (threadIdx.x & (32 - kLanes));
#pragma unroll
  for (int o = kLanes / 2; o > 0; o >>= 1) s += __shfl_xor_sync(grp, s, o);
  return s;
}

__global__ void k_apply_t(const long long* __restrict__ rowptr, const int* __restrict__ col,
                          const float* __restrict__ val, const float* __restrict__ x, float* y,
                          long long len) {
  const long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / kLanes;
  const int lane = threadIdx.x % kLanes;
  if (row >= len) return;
  const float s = row_dot(rowptr, col, val, x, row, lane);
  if (lane == 0) y[row] = s;
}

struct W7 { float w[7]; };

__device__ __forceinline__ long long iface_index(const SetLayout& L, int f, int ix) {
  return f < 3 ? L.off[f] + (long long)(L.nzf - 1) * L.pitch[f] + ix : L.off[f] + ix;
}

constexpr int kStartThreads = 128;                    // columns of transposed averages per block
constexpr int kStartCols = kStartThreads - 6;         // output columns per block (3-column halos)

// The start of one transposed step over the interface columns 3..nx-4, with
// the smoothing halos recomputed per block (no grid-wide barrier):
//   v_f(ix)   = lam_f(ix) (+ the step's residual on svx, svz, fp when res != null)
//   tmp_f(ix) = (A^T v)_f (ix) / wsum(ix)          A: the continuity average
//   s_f(j)    = sum_k w_k tmp_f(j - k), k = -3..3  (only ix in 3..nx-4)
// s goes to mu and to kb = c M s; lam itself is only read (the step's first
// transposed stage takes its lam from mu, where mu = lam off these cells).
// Receivers sample the filtered interface rows of columns 3..nx-4 only, so the
// residuals enter there (elsewhere the record is 0 whatever the state).
// Threads (column t, field f): blockDim = (kStartThreads, 8).
__global__ void __launch_bounds__(kStartThreads * 8) k_step_start(
    const float* __restrict__ lam, SetLayout L, const float2* __restrict__ nrm, W7 w7,
    const float* __restrict__ res, float* mu, float* kb, const uint8_t* __restrict__ mask, float c) {
  __shared__ float tmp[8][kStartThreads];
  const int nx = L.nx, f = threadIdx.y;
  const int ix = blockIdx.x * kStartCols + threadIdx.x;  // = output column j0 - 3 + threadIdx.x
  if (ix >= 3 && ix <= nx - 4) {
    float lv[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) lv[q] = lam[iface_index(L, q, ix)];
    if (res) {
      lv[3] += __ldg(res + ix);
      lv[4] += __ldg(res + nx + ix);
      lv[2] += __ldg(res + 2 * nx + ix);
    }
    const int klo = max(-3, 3 - ix), khi = min(3, nx - 4 - ix);
    float wsum = 0.0f;
    for (int k = klo; k <= khi; ++k) wsum += w7.w[k + 3];
    const float2 n = __ldg(nrm + ix);
    float e[8], u[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) e[q] = q == f ? 1.0f : 0.0f;
    interface_average(n, e, u);
    float t = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q) t = fmaf(lv[q], u[q], t);
    tmp[f][threadIdx.x] = t / wsum;
  }
  __syncthreads();
  if (threadIdx.x < 3 || threadIdx.x >= kStartThreads - 3 || ix < 3 || ix > nx - 4) return;
  float s = 0.0f;
#pragma unroll
  for (int k = -3; k <= 3; ++k) {
    const int i = ix - k;
    if (i >= 3 && i <= nx - 4) s = fmaf(w7.w[k + 3], tmp[f][threadIdx.x - k], s);
  }
  const long long q = iface_index(L, f, ix);
  mu[q] = s;
  kb[q] = mask[q] ? c * s : 0.0f;
}


__global__ void k_drop_count(const long long* __restrict__ rowptr, const int* __restrict__ col,
                             SetLayout L, unsigned long long* count) {
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= L.len) return;
  unsigned long long n = 0;
  for (long long k = rowptr[j]; k < rowptr[j + 1]; ++k) {
    int a, r, c;
    if (!(locate(L, col[k], a, r, c) && structured_cell(L, a, r, c))) ++n;
  }
  count[j] = n;
}

__global__ void k_drop_fill(const long long* __restrict__ rowptr, const int* __restrict__ col,
                            const float* __restrict__ val, SetLayout L,
                            const long long* __restrict__ rp2, int* col2, float* val2) {
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= L.len) return;
  long long o = rp2[j];
  for (long long k = rowptr[j]; k < rowptr[j + 1]; ++k) {
    int a, r, c;
    if (!(locate(L, col[k], a, r, c) && structured_cell(L, a, r, c))) {
      col2[o] = col[k];
      val2[o] = val[k];
      ++o;
    }
  }
}

// Q fields of the transposed interior formulas at every main-field cell (0
// outside the interior set). For an interior output cell i the forward stage is
// (pml_fs_kernels.cuh:333-752, interior branches)
//   fluid  k_vx = -r (xix Dx p + zex Dz p),  k_vz = -r (xiz Dx p + zez Dz p),
//          k_p  = -K (xix Dx vx + zex Dz vx + xiz Dx vz + zez Dz vz)
//   solid  k_vx = r (xix Dx sx + zex Dz sx + xiz Dx sxz + zez Dz sxz),
//          k_vz = r (xix Dx sxz + zex Dz sxz + xiz Dx sz + zez Dz sz),
//          k_sx = c11 (xix Dx vx + zex Dz vx) + c13 (xiz Dx vz + zez Dz vz),
//          k_sz = c13 (xix Dx vx + zex Dz vx) + c33 (xiz Dx vz + zez Dz vz),
//          k_sxz = c55 (xiz' Dx vx + zez' Dz vx + xix' Dx vz + zex' Dz vz)
// (r = 1/rho; the primed metric is read at global row iz in the four-side CPML
// variant, cpml_kernels.cuh:448-455), so the Dx / Dz coefficient of every
// (output, input) pair times x at i, summed per input field, gives qx / qz.
// Transposes of the stage right-hand side at a PML strip cell of a structured
// row. There the right-hand side is linear in the cell's biased derivatives
// and ADE memory (fluid_rhs / solid_rhs, the branches without the conservative
// form); given the stage adjoint y of the cell's outputs these return the
// adjoint of every input, i.e. the cell's Q-field entries and the point-wise
// ADE transpose. R = gxz / gxx and S = gxz / gzz as in the forward.
//
// Fluid: y = (vx, vz, p, xi Vx, Vz, Ex, Ez) outputs; d = adjoint of
// (Dx p, Dz p, Dx vx, Dz vx, Dx vz, Dz vz), e = adjoint of the xi ADE (Vx, Vz, Ex, Ez).
template <bool CPML>
__device__ __forceinline__ void fluid_strip_t(const float* y, float xix, float xiz, float zex,
                                              float zez, float rr, float K, float4 pml, float* d,
                                              float* e) {
  const float gxx = xix * xix + xiz * xiz, gxz = xix * zex + xiz * zez, R = gxz / gxx;
  const float dpb = pml.x, apdpb = pml.y, invb = pml.z;
  // momentum: vx, vz and the Vx, Vz memory read divx, divz = -(xix, xiz) (Dx p + R Dz p)
  const float gdx = rr * (invb - 1.0f) * y[0] + dpb * y[3];
  const float gdz = rr * (invb - 1.0f) * y[1] + dpb * y[4];
  const float gdiv = -(xix * gdx + xiz * gdz);
  d[0] = -rr * (xix * y[0] + xiz * y[1]) + gdiv;
  d[1] = -rr * (zex * y[0] + zez * y[1]) + R * gdiv;
  e[0] = -rr * invb * y[0] - apdpb * y[3];
  e[1] = -rr * invb * y[1] - apdpb * y[4];
  // pressure: p and the Ex, Ez memory read Dvx = Dx vx + R Dz vx, Dvz likewise
  const float gDvx = -K * (invb - 1.0f) * xix * y[2] + dpb * y[5];
  const float gDvz = -K * (invb - 1.0f) * xiz * y[2] + dpb * y[6];
  d[2] = -K * xix * y[2] + gDvx;
  d[3] = -K * zex * y[2] + R * gDvx;
  d[4] = -K * xiz * y[2] + gDvz;
  d[5] = -K * zez * y[2] + R * gDvz;
  e[2] = K * invb * xix * y[2] - apdpb * y[5];
  e[3] = K * invb * xiz * y[2] - apdpb * y[6];
}

// Solid: y = (vx, vz, sx, sz, sxz, xi Vx, Vz, Ex, Ez, zeta Vx, Vz, Ex, Ez);
// d = adjoint of (Dx sx, Dz sx, Dx sz, Dz sz, Dx sxz, Dz sxz, Dx vx, Dz vx,
// Dx vz, Dz vz); e = adjoint of the xi then the zeta ADE (Vx, Vz, Ex, Ez).
// The sxz line's own metric (bxix ..) differs from the cell's only in the
// four-side CPML variant (cpml_kernels.cuh:448-455); its PML terms use the cell's.
struct SolidCell {
  float xix, xiz, zex, zez, bxix, bxiz, bzex, bzez, rr, c11, c13, c33, c55;
  float4 px, pz;
  bool side, bottom;
};

__device__ __forceinline__ void solid_strip_t(const float* y, const SolidCell& k, float* d,
                                              float* e) {
  const float xix = k.xix, xiz = k.xiz, zex = k.zex, zez = k.zez;
  const float gxx = xix * xix + xiz * xiz, gzz = zex * zex + zez * zez, gxz = xix * zex + xiz * zez;
  const float R = gxz / gxx, S = gxz / gzz;
  const float gvx = k.rr * y[0], gvz = k.rr * y[1];
  // momentum: rho v_t = div sigma (+ the projected PML terms dxx, dxz, dzx, dzz)
  float gxx_ = 0.f, gxz_ = 0.f, gzx_ = 0.f, gzz_ = 0.f;
  for (int q = 0; q < 8; ++q) e[q] = 0.0f;
  if (k.side) {
    const float dp = k.px.x, ap = k.px.y, ib = k.px.z;
    gxx_ = k.rr * (ib - 1.0f) * y[0] + dp * y[5];
    gxz_ = k.rr * (ib - 1.0f) * y[1] + dp * y[6];
    e[0] = -k.rr * ib * y[0] - ap * y[5];
    e[1] = -k.rr * ib * y[1] - ap * y[6];
  }
  if (k.bottom) {
    const float dq = k.pz.x, aq = k.pz.y, jb = k.pz.z;
    gzx_ = k.rr * (jb - 1.0f) * y[0] + dq * y[9];
    gzz_ = k.rr * (jb - 1.0f) * y[1] + dq * y[10];
    e[4] = -k.rr * jb * y[0] - aq * y[9];
    e[5] = -k.rr * jb * y[1] - aq * y[10];
  }
  // dxx = xix (sxdx + R sxdz) + xiz (tdx + R tdz); dxz = xix (tdx + R tdz) + xiz (szdx + R szdz)
  // dzx = zex (sxdz + S sxdx) + zez (S tdx + tdz); dzz = zex (S tdx + tdz) + zez (S szdx + szdz)
  d[0] = gvx * xix + gxx_ * xix + S * gzx_ * zex;
  d[1] = gvx * zex + R * gxx_ * xix + gzx_ * zex;
  d[2] = gvz * xiz + gxz_ * xiz + S * gzz_ * zez;
  d[3] = gvz * zez + R * gxz_ * xiz + gzz_ * zez;
  d[4] = gvx * xiz + gvz * xix + gxx_ * xiz + gxz_ * xix + S * (gzx_ * zez + gzz_ * zex);
  d[5] = gvx * zez + gvz * zex + R * (gxx_ * xiz + gxz_ * xix) + gzx_ * zez + gzz_ * zex;
  // stress: the constitutive law and its projected PML terms
  const float c11 = k.c11, c13 = k.c13, c33 = k.c33, c55 = k.c55;
  float vxdx = (c11 * y[2] + c13 * y[3]) * xix + c55 * k.bxiz * y[4];
  float vxdz = (c11 * y[2] + c13 * y[3]) * zex + c55 * k.bzez * y[4];
  float vzdx = (c13 * y[2] + c33 * y[3]) * xiz + c55 * k.bxix * y[4];
  float vzdz = (c13 * y[2] + c33 * y[3]) * zez + c55 * k.bzex * y[4];
  if (k.side) {
    const float dp = k.px.x, ap = k.px.y, ib = k.px.z;
    const float ax = (c11 * y[2] + c13 * y[3]) * xix + c55 * xiz * y[4];
    const float az = (c13 * y[2] + c33 * y[3]) * xiz + c55 * xix * y[4];
    const float gDvx = (ib - 1.0f) * ax + dp * y[7], gDvz = (ib - 1.0f) * az + dp * y[8];
    vxdx += gDvx;
    vxdz += R * gDvx;
    vzdx += gDvz;
    vzdz += R * gDvz;
    e[2] = -ib * ax - ap * y[7];
    e[3] = -ib * az - ap * y[8];
  }
  if (k.bottom) {
    const float dq = k.pz.x, aq = k.pz.y, jb = k.pz.z;
    const float bx = (c11 * y[2] + c13 * y[3]) * zex + c55 * zez * y[4];
    const float bz = (c13 * y[2] + c33 * y[3]) * zez + c55 * zex * y[4];
    const float gFvx = (jb - 1.0f) * bx + dq * y[11], gFvz = (jb - 1.0f) * bz + dq * y[12];
    vxdz += gFvx;
    vxdx += S * gFvx;
    vzdz += gFvz;
    vzdx += S * gFvz;
    e[6] = -jb * bx - aq * y[11];
    e[7] = -jb * bz - aq * y[12];
  }
  d[6] = vxdx;
  d[7] = vxdz;
  d[8] = vzdx;
  d[9] = vzdz;
}

// Q fields of fluid cell (r, c); only structured cells are non-zero. A strip
// cell also writes the point-wise transpose of its ADE inputs into t (those
// rows have no CSR entries: every output that reads them is at this cell).
template <bool CPML>
__device__ __forceinline__ void q_fluid(const Coef& C, const SetLayout& L, const float* __restrict__ x,
                                        float* qx, float* qz, float* t, int r, int c,
                                        bool write_zero) {
  const size_t g = (size_t)r * C.P + c;
  const long long i0 = L.off[0] + g, i1 = L.off[1] + g, i2 = L.off[2] + g;
  if (!structured_cell(L, 0, r, c)) {
    if (write_zero) {
      qx[i0] = 0.f; qz[i0] = 0.f; qx[i1] = 0.f; qz[i1] = 0.f; qx[i2] = 0.f; qz[i2] = 0.f;
    }
    return;
  }
  const float xix = __ldg(C.xix + g), xiz = __ldg(C.xiz + g), zex = __ldg(C.zex + g),
              zez = __ldg(C.zez + g), rr = __ldg(C.rhof + g), K = __ldg(C.K + g);
  const float kvx = x[i0], kvz = x[i1], kp = x[i2];
  const int s = col_to_strip(c, L.nx, L.npd);
  if (s < 0) {
    qx[i2] = -rr * (xix * kvx + xiz * kvz);
    qz[i2] = -rr * (zex * kvx + zez * kvz);
    qx[i0] = -K * xix * kp;
    qz[i0] = -K * zex * kp;
    qx[i1] = -K * xiz * kp;
    qz[i1] = -K * zez * kp;
    return;
  }
  const float4 pml = __ldg(C.pmlx + c);
  long long ia[4];
  float y[7] = {kvx, kvz, kp, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    ia[q] = L.off[8 + q] + (long long)r * L.pitch[8 + q] + s;
    y[3 + q] = x[ia[q]];
  }
  float dq[6], eq[4];
  fluid_strip_t<CPML>(y, xix, xiz, zex, zez, rr, K, pml, dq, eq);
  qx[i2] = dq[0];
  qz[i2] = dq[1];
  qx[i0] = dq[2];
  qz[i0] = dq[3];
  qx[i1] = dq[4];
  qz[i1] = dq[5];
  if (t) {
#pragma unroll
    for (int q = 0; q < 4; ++q) t[ia[q]] = eq[q];
  }
}

// Q fields of solid cell (r, c); only structured cells are non-zero. Strip and
// bottom-band cells also write the point-wise transpose of their ADE inputs into t.
template <bool CPML>
__device__ __forceinline__ void q_solid(const Coef& C, const SetLayout& L, const float* __restrict__ x,
                                        float* qx, float* qz, float* t, int r, int c,
                                        bool write_zero) {
  const int P = C.P;
  const size_t m = (size_t)r * P + c, g = m + (size_t)(L.nzf - 1) * P;
  float q[10] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // (x, z) for vx, vz, sx, sz, sxz
  if (structured_cell(L, 3, r, c)) {
    const float xix = __ldg(C.xix + g), xiz = __ldg(C.xiz + g), zex = __ldg(C.zex + g),
                zez = __ldg(C.zez + g);
    const size_t b = CPML ? m : g;
    const float bxix = __ldg(C.xix + b), bxiz = __ldg(C.xiz + b), bzex = __ldg(C.zex + b),
                bzez = __ldg(C.zez + b);
    const float rr = __ldg(C.rhos + m), c11 = __ldg(C.C11 + m), c13 = __ldg(C.C13 + m),
                c33 = __ldg(C.C33 + m), c55 = __ldg(C.C55 + m);
    const float kvx = x[L.off[3] + m], kvz = x[L.off[4] + m], ksx = x[L.off[5] + m],
                ksz = x[L.off[6] + m], ksxz = x[L.off[7] + m];
    const int s = col_to_strip(c, L.nx, L.npd), zb0 = L.nzs - 3 - L.npd;
    if (s < 0 && r < zb0) {
      const float a1 = c11 * ksx + c13 * ksz, a2 = c13 * ksx + c33 * ksz;
      q[0] = xix * a1 + c55 * bxiz * ksxz;   // vx, x
      q[1] = zex * a1 + c55 * bzez * ksxz;   // vx, z
      q[2] = xiz * a2 + c55 * bxix * ksxz;   // vz, x
      q[3] = zez * a2 + c55 * bzex * ksxz;   // vz, z
      q[4] = rr * xix * kvx;                 // sx
      q[5] = rr * zex * kvx;
      q[6] = rr * xiz * kvz;                 // sz
      q[7] = rr * zez * kvz;
      q[8] = rr * (xiz * kvx + xix * kvz);   // sxz
      q[9] = rr * (zez * kvx + zex * kvz);
    } else {
      SolidCell k{xix, xiz, zex, zez, bxix, bxiz, bzex, bzez, rr, c11, c13, c33, c55,
                  make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f), s >= 0, r >= zb0};
      if (k.side) k.px = __ldg(C.pmlx + c);
      if (k.bottom) k.pz = __ldg(C.pmlz + r);
      long long ia[8];
      float y[13] = {kvx, kvz, ksx, ksz, ksxz, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        ia[u] = k.side ? L.off[12 + u] + (long long)r * L.pitch[12 + u] + s : -1;
        ia[4 + u] = k.bottom ? L.off[16 + u] + (long long)(r - zb0) * L.pitch[16 + u] + c : -1;
        y[5 + u] = k.side ? x[ia[u]] : 0.f;
        y[9 + u] = k.bottom ? x[ia[4 + u]] : 0.f;
      }
      float dq[10], eq[8];
      solid_strip_t(y, k, dq, eq);
      // d order: sx, sz, sxz (x, z) then vx, vz (x, z); q order: vx, vz, sx, sz, sxz (x, z)
      q[4] = dq[0]; q[5] = dq[1]; q[6] = dq[2]; q[7] = dq[3]; q[8] = dq[4]; q[9] = dq[5];
      q[0] = dq[6]; q[1] = dq[7]; q[2] = dq[8]; q[3] = dq[9];
      if (t) {
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (ia[u] >= 0) t[ia[u]] = eq[u];
      }
    }
  } else if (!write_zero) {
    return;
  }
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    qx[L.off[3 + f] + m] = q[2 * f];
    qz[L.off[3 + f] + m] = q[2 * f + 1];
  }
}

// ZERO: also write the zeros off the interior cells (a fresh Q buffer).
template <bool CPML, bool ZERO = true>
__global__ void k_qfields(Coef C, SetLayout L, const float* __restrict__ x, float* qx, float* qz,
                          float* t) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (c >= L.nx) return;
  if (row < L.nzf) q_fluid<CPML>(C, L, x, qx, qz, t, row, c, ZERO);
  else q_solid<CPML>(C, L, x, qx, qz, t, row - L.nzf, c, ZERO);
}

// The Q fields of x (the grid rows below nz_f + nz_s, as k_qfields without
// zeroing) and, in the grid rows after them, the probed sparse rows of L^T x
// into t (kLanes threads a row), in one launch: both only read x, and they
// write disjoint rows of t (the ADE rows of structured cells, the rows with
// entries).
template <bool CPML>
__global__ void k_prepare(Coef C, SetLayout L, const float* __restrict__ x, float* qx, float* qz,
                          float* t, const int* __restrict__ nzrow,
                          const long long* __restrict__ rowptr, const int* __restrict__ col,
                          const float* __restrict__ val, long long nrows) {
  const int row = blockIdx.y, nq = L.nzf + L.nzs;
  if (row < nq) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= L.nx) return;
    if (row < L.nzf) q_fluid<CPML>(C, L, x, qx, qz, t, row, c, false);
    else q_solid<CPML>(C, L, x, qx, qz, t, row - L.nzf, c, false);
    return;
  }
  const long long g = ((long long)(row - nq) * gridDim.x + blockIdx.x) * blockDim.x + threadIdx.x;
  const long long r = g / kLanes;
  const int lane = threadIdx.x % kLanes;
  if (r >= nrows) return;  // whole groups leave together
  const int j = nzrow[r];
  const float sum = row_dot(rowptr, col, val, x, j, lane);
  if (lane == 0) t[j] = sum;
}

// ---- material gradients ----------------------------------------------------------

struct Grad {
  double *K, *rf, *c11, *c13, *c33, *c55, *rs;
};

template <int DIR, bool CPML>
__device__ __forceinline__ void grad_iface(const Coef& C, const Fields& Y, const Fields& KB,
                                           const Grad& G, int ix);

// blockIdx.y = 0: the interface columns (first, they take longest); then fluid
// rows 3..nz_f-2 and solid rows 1..nz_s-4; columns 3..nx-4. Interior cells also
// write the Q fields of the stage adjoint (kb) for the transposed operator.
template <int DIR, bool CPML>
__global__ void __launch_bounds__(128, 6) k_grad_cells(Coef C, SetLayout L, Fields Y, Fields KB,
                                                    const float* __restrict__ kb, float* qx,
                                                    float* qz, Grad G) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = C.nx, P = C.P, nzf = C.nzf, nzs = C.nzs, npd = C.npd;
  if (ix < 3 || ix > nx - 4) return;
  if (blockIdx.y == 0) {
    grad_iface<DIR, CPML>(C, Y, KB, G, ix);
    return;
  }
  const bool side = min(ix - 3, nx - 4 - ix) < npd;
  const int scol = side ? xstrip_col(ix, nx, npd) : 0;
  const int nfr = nzf - 4;
  const int row = blockIdx.y - 1;
  if (row < nfr) {
    const int iz = 3 + row;
    const size_t g = (size_t)iz * P + ix;
    // the accumulated gradients first: their loads must not wait for a store
    // (the pointers may alias as far as the compiler knows)
    const double grf = G.rf[g], gK = G.K[g];
    float ade[4] = {0.f, 0.f, 0.f, 0.f}, zade[4] = {0.f, 0.f, 0.f, 0.f};
    if (side)
      for (int q = 0; q < 4; ++q) ade[q] = __ldg(Y.fx[q] + (size_t)iz * C.Ps + scol);
    const bool top = CPML && iz <= npd + 2;
    if (top)
      for (int q = 0; q < 4; ++q) zade[q] = __ldg(Y.fz[q] + (size_t)(iz - 3) * P + ix);
    const FluidCoefs cf{__ldg(C.xix + g), __ldg(C.xiz + g), __ldg(C.zex + g), __ldg(C.zez + g),
                        1.0f, 1.0f};
    FluidGlobal A{Y.fvx, Y.fvz, Y.fp, g, P};
    const FluidK o = fluid_rhs<DIR, false, CPML>(C, A, iz, ix, side, ade, cf, top, zade);
    // velocity terms carry 1/rho, the pressure term K
    G.rf[g] = grf + (double(__ldg(KB.fvx + g)) * o.vx + double(__ldg(KB.fvz + g)) * o.vz);
    G.K[g] = gK + double(__ldg(KB.fp + g)) * o.p;
    if (qx) q_fluid<CPML>(C, L, kb, qx, qz, nullptr, iz, ix, false);
    return;
  }
  const int iz = 1 + row - nfr;
  if (iz > nzs - 4) return;
  const size_t m = (size_t)iz * P + ix, g = m + (size_t)(nzf - 1) * P;
  const int zb0 = nzs - 3 - npd;
  const bool bottom = iz >= zb0;
  const double gc11 = G.c11[m], gc33 = G.c33[m], gc55 = G.c55[m], grs = G.rs[m], gc13 = G.c13[m];
  float xade[4] = {0.f, 0.f, 0.f, 0.f}, zade[4] = {0.f, 0.f, 0.f, 0.f};
  if (side)
    for (int q = 0; q < 4; ++q) xade[q] = __ldg(Y.sx[q] + (size_t)iz * C.Ps + scol);
  if (bottom)
    for (int q = 0; q < 4; ++q) zade[q] = __ldg(Y.sz[q] + (size_t)(iz - zb0) * P + ix);
  const float xix = __ldg(C.xix + g), xiz = __ldg(C.xiz + g), zex = __ldg(C.zex + g),
              zez = __ldg(C.zez + g);
  SolidGlobal A{Y.svx, Y.svz, Y.ssx, Y.ssz, Y.ssxz, m, P};
  const double kvx = __ldg(KB.svx + m), kvz = __ldg(KB.svz + m), ksx = __ldg(KB.ssx + m),
               ksz = __ldg(KB.ssz + m), ksxz = __ldg(KB.ssxz + m);
  // C11, C33, C55 and 1/rho each reach a different output; C13 reaches sx and sz
  const SolidK o1 = solid_rhs<DIR, false, CPML>(C, A, iz, ix, side, bottom, xade, zade,
                                                SolidCoefs{xix, xiz, zex, zez, 1.f, 1.f, 0.f, 1.f, 1.f});
  double t13;
  if (!side && !bottom) {
    // off the PML strips the stress RHS is sx = C11 X + C13 Z, sz = C13 X + C33 Z,
    // so the unit-C13 outputs (Z, X) are the unit-C11/C33 ones swapped
    t13 = ksx * o1.sz + ksz * o1.sx;
  } else {
    const SolidK o2 = solid_rhs<DIR, false, CPML>(C, A, iz, ix, side, bottom, xade, zade,
                                                  SolidCoefs{xix, xiz, zex, zez, 0.f, 0.f, 1.f, 0.f, 0.f});
    t13 = ksx * o2.sx + ksz * o2.sz;
  }
  G.c11[m] = gc11 + ksx * o1.sx;
  G.c33[m] = gc33 + ksz * o1.sz;
  G.c55[m] = gc55 + ksxz * o1.sxz;
  G.rs[m] = grs + (kvx * o1.vx + kvz * o1.vz);
  G.c13[m] = gc13 + t13;
  if (qx) q_solid<CPML>(C, L, kb, qx, qz, nullptr, iz, ix, false);
}

// Interface column ix: both media's RHS at the interface row, coupled, per coefficient.
template <int DIR, bool CPML>
__device__ __forceinline__ void grad_iface(const Coef& C, const Fields& Y, const Fields& KB,
                                           const Grad& G, int ix) {
  const int nx = C.nx, P = C.P, nzf = C.nzf, nzs = C.nzs, npd = C.npd;
  const bool side = min(ix - 3, nx - 4 - ix) < npd;
  const int scol = side ? xstrip_col(ix, nx, npd) : 0;
  const int zb0 = nzs - 3 - npd;
  const bool bottom = 0 >= zb0;
  const bool ftop = CPML && nzf - 1 <= npd + 2;
  const size_t fi = (size_t)(nzf - 1) * P + ix, si = ix, gs = si + (size_t)(nzf - 1) * P;
  float fade[4] = {0.f, 0.f, 0.f, 0.f}, xade[4] = {0.f, 0.f, 0.f, 0.f},
        zade[4] = {0.f, 0.f, 0.f, 0.f}, ztop[4] = {0.f, 0.f, 0.f, 0.f};
  if (side)
    for (int q = 0; q < 4; ++q) {
      fade[q] = __ldg(Y.fx[q] + (size_t)(nzf - 1) * C.Ps + scol);
      xade[q] = __ldg(Y.sx[q] + scol);
    }
  if (bottom)
    for (int q = 0; q < 4; ++q) zade[q] = __ldg(Y.sz[q] + (size_t)(0 - zb0) * P + ix);
  if (ftop)
    for (int q = 0; q < 4; ++q) ztop[q] = __ldg(Y.fz[q] + (size_t)(nzf - 1 - 3) * P + ix);
  FluidGlobal Af{Y.fvx, Y.fvz, Y.fp, fi, P};
  SolidGlobal As{Y.svx, Y.svz, Y.ssx, Y.ssz, Y.ssxz, si, P};
  const float fxix = __ldg(C.xix + fi), fxiz = __ldg(C.xiz + fi), fzex = __ldg(C.zex + fi),
              fzez = __ldg(C.zez + fi);
  const float sxix = __ldg(C.xix + gs), sxiz = __ldg(C.xiz + gs), szex = __ldg(C.zex + gs),
              szez = __ldg(C.zez + gs);
  const FluidK of = fluid_rhs<DIR, false, CPML>(C, Af, nzf - 1, ix, side, fade,
                                                FluidCoefs{fxix, fxiz, fzex, fzez, 1.f, 1.f}, ftop, ztop);
  const SolidK o1 = solid_rhs<DIR, false, CPML>(C, As, 0, ix, side, bottom, xade, zade,
                                                SolidCoefs{sxix, sxiz, szex, szez, 1.f, 1.f, 0.f, 1.f, 1.f});
  const SolidK o2 = solid_rhs<DIR, false, CPML>(C, As, 0, ix, side, bottom, xade, zade,
                                                SolidCoefs{sxix, sxiz, szex, szez, 0.f, 0.f, 1.f, 0.f, 0.f});
  const float kb[8] = {__ldg(KB.fvx + fi), __ldg(KB.fvz + fi), __ldg(KB.fp + fi), __ldg(KB.svx + si),
                       __ldg(KB.svz + si), __ldg(KB.ssx + si), __ldg(KB.ssz + si), __ldg(KB.ssxz + si)};
  const float2 n = __ldg(C.nrm + ix);
  // one coefficient at a time: its own outputs before the coupling, the rest 0
  auto coupled = [&](float f0, float f1, float f2, float s0, float s1, float s2, float s3,
                     float s4) -> double {
    const float kf[3] = {f0, f1, f2}, ks[5] = {s0, s1, s2, s3, s4};
    float kv[8];
    couple_rhs<DIR>(n, kf, ks, kv);
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) t += double(kb[q]) * kv[q];
    return t;
  };
  G.rf[fi] += coupled(of.vx, of.vz, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f);
  G.K[fi] += coupled(0.f, 0.f, of.p, 0.f, 0.f, 0.f, 0.f, 0.f);
  G.rs[si] += coupled(0.f, 0.f, 0.f, o1.vx, o1.vz, 0.f, 0.f, 0.f);
  G.c11[si] += coupled(0.f, 0.f, 0.f, 0.f, 0.f, o1.sx, 0.f, 0.f);
  G.c33[si] += coupled(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, o1.sz, 0.f);
  G.c55[si] += coupled(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, o1.sxz);
  G.c13[si] += coupled(0.f, 0.f, 0.f, 0.f, 0.f, o2.sx, o2.sz, 0.f);
}

// Transposed interior stencil at element j of a main array (row r of `rows`,
// column c of nx, pitch P), addressed relative to j: D_F^T g (j) =
// sum_t a_t g(j - t), D_B^T g (j) = -sum_t a_t g(j + t), taps t = -1..3 of
// the DRP pair, along x in qx and along z in qz. CHECK: taps may leave the array.
template <int DIR, bool CHECK>
__device__ __forceinline__ float t_stencil(const float* __restrict__ qx, const float* __restrict__ qz,
                                           long long j, int r, int c, int P, int rows, int nx) {
  const float at[5] = {kAm1, kA0, kA1, kA2, kA3};
  float s = 0.0f;
#pragma unroll
  for (int t = -1; t <= 3; ++t) {
    const int d = DIR == kDirF ? -t : t;
    if (!CHECK || (c + d >= 0 && c + d < nx)) s = fmaf(at[t + 1], __ldg(qx + j + d), s);
    if (!CHECK || (r + d >= 0 && r + d < rows))
      s = fmaf(at[t + 1], __ldg(qz + j + (long long)d * P), s);
  }
  return DIR == kDirF ? s : -s;
}

constexpr int kRevBlock = 128;
constexpr int kRevVec = 4;  // consecutive elements per thread

// The RK bookkeeping of one element of a reverse stage (see k_reverse_h).
template <int MODE>
__device__ __forceinline__ void rev_finish(float y, float lam0, float mu0, bool mk, float w,
                                           float cw, bool has_kbn, float& lam, float& mu_out,
                                           float& kbn_out) {
  if (MODE == 0) {
    lam = y;
    return;
  }
  const float m = mk ? 1.0f : 0.0f;
  if (MODE == 1) {
    lam = lam0 + y;
    if (has_kbn) {
      mu_out = lam;
      kbn_out = mk ? w * lam : 0.0f;
    }
    return;
  }
  lam = lam0 + m * y;
  if (MODE == 2 || MODE == 4) kbn_out = m * fmaf(cw, y, w * mu0);
}

// One element, scalar loads (edges, padding and the rest of the set).
// stencil: a main-array element at row r of `rows`, column c < nx.
template <int DIR, int MODE>
__device__ __forceinline__ void rev_one(const float* __restrict__ t, const float* __restrict__ qx,
                                        const float* __restrict__ qz, long long j, bool stencil,
                                        int r, int c, int P, int rows, int nx, float* y_or_lam,
                                        const uint8_t* __restrict__ mask, float* kbn, float* mu,
                                        float w, float cw) {
  float y = t[j];
  // the RK operands first: their loads must not wait for a store
  const float mu0 = (MODE == 2 || MODE == 4) ? mu[j] : 0.f;
  const float lam0 = MODE == 0 ? 0.f : (MODE == 4 ? mu0 : y_or_lam[j]);
  const bool mk = MODE == 0 ? false : mask[j] != 0;
  if (stencil) {
    if (c >= 3 && c <= nx - 4 && r >= 3 && r <= rows - 4)
      y += t_stencil<DIR, false>(qx, qz, j, r, c, P, rows, nx);
    else
      y += t_stencil<DIR, true>(qx, qz, j, r, c, P, rows, nx);
  }
  float lam = 0.f, mo = 0.f, ko = 0.f;
  rev_finish<MODE>(y, lam0, mu0, mk, w, cw, kbn != nullptr, lam, mo, ko);
  y_or_lam[j] = lam;
  if (MODE == 1 && kbn) {
    mu[j] = mo;
    kbn[j] = ko;
  }
  if (MODE == 2 || MODE == 4) kbn[j] = ko;
}

__device__ __forceinline__ float f4(const float4& v, int k) {
  return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}

// One thread per kRevVec consecutive rows of L^T (j0 a multiple of kRevVec):
// the sparse rest plus, on main-field cells, the transposed interior stencil;
// then the RK bookkeeping of the reverse stage.
// MODE 0: y only; 1: lam += y and, with kbn, the start of the next transposed
// step: mu = lam, kbn = w M lam; 2: lam += M y, kbn = M (w mu + c y); 3: lam += M y;
// 4: MODE 2 with lam taken from mu (the step's first stage: the step start
// wrote the filtered interface cells to mu only, and mu = lam elsewhere).
// `t` holds the CSR part of every row (k_rows_csr; rows without entries keep 0).
// Grid: x over the pitch P of the main arrays (kRevVec columns a thread);
// z < 8: main array z (the fluid block [3][nz_f][P] at 0, the solid block
// [5][nz_s][P] at off[3]), y its row; z = 8: the rest of the set from `tail0`
// in runs of gridDim.x * kRevBlock * kRevVec elements (strips, bands,
// padding), striding by gridDim.y. Four columns whose stencils stay inside the
// array take 16-byte loads and stores (every row starts 16-byte aligned: P
// and the array offsets are multiples of 32 floats), with the taps of each
// column summed in the same order as the scalar path.
template <int DIR, int MODE>
__global__ void __launch_bounds__(kRevBlock) k_reverse_h(
    const float* __restrict__ t, const float* __restrict__ qx, const float* __restrict__ qz,
    SetLayout L, long long tail0, float* y_or_lam, const uint8_t* __restrict__ mask, float* kbn,
    float* mu, float w, float cw) {
  const int a = blockIdx.z;
  const int P = L.pitch[0], nx = L.nx;
  if (a < 8) {
    const bool fluid = a < 3;
    const int rows = fluid ? L.nzf : L.nzs;
    const int r = blockIdx.y, c0 = (blockIdx.x * kRevBlock + threadIdx.x) * kRevVec;
    if (r >= rows || c0 >= P) return;
    const long long j0 = fluid ? (long long)(a * L.nzf + r) * P + c0
                               : L.off[3] + (long long)((a - 3) * L.nzs + r) * P + c0;
    if (c0 >= 4 && c0 + kRevVec - 1 <= nx - 4 && r >= 3 && r <= rows - 4) {
      const float4 tv = *reinterpret_cast<const float4*>(t + j0);
      float4 lv = make_float4(0.f, 0.f, 0.f, 0.f), mv = lv;
      uchar4 kv = make_uchar4(0, 0, 0, 0);
      if (MODE == 2 || MODE == 4) mv = *reinterpret_cast<const float4*>(mu + j0);
      if (MODE == 1 || MODE == 2 || MODE == 3) lv = *reinterpret_cast<const float4*>(y_or_lam + j0);
      if (MODE == 4) lv = mv;
      if (MODE != 0) kv = *reinterpret_cast<const uchar4*>(mask + j0);
      // qx along the row: elements j0 - 4 .. j0 + 7 cover the taps of all four columns
      const float4 xa = __ldg(reinterpret_cast<const float4*>(qx + j0 - 4));
      const float4 xb = __ldg(reinterpret_cast<const float4*>(qx + j0));
      const float4 xc = __ldg(reinterpret_cast<const float4*>(qx + j0 + 4));
      float4 zr[5];
#pragma unroll
      for (int t5 = -1; t5 <= 3; ++t5) {
        const int d = DIR == kDirF ? -t5 : t5;
        zr[t5 + 1] = __ldg(reinterpret_cast<const float4*>(qz + j0 + (long long)d * P));
      }
      const float at[5] = {kAm1, kA0, kA1, kA2, kA3};
      float yo[4], lo[4], mo[4], ko[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        float sum = 0.0f;
#pragma unroll
        for (int t5 = -1; t5 <= 3; ++t5) {
          const int d = DIR == kDirF ? -t5 : t5;
          const int q = k + d + 4;  // index in xa|xb|xc
          const float xv = q < 4 ? f4(xa, q) : (q < 8 ? f4(xb, q - 4) : f4(xc, q - 8));
          sum = fmaf(at[t5 + 1], xv, sum);
          sum = fmaf(at[t5 + 1], f4(zr[t5 + 1], k), sum);
        }
        yo[k] = f4(tv, k) + (DIR == kDirF ? sum : -sum);
        const unsigned char mb = k == 0 ? kv.x : (k == 1 ? kv.y : (k == 2 ? kv.z : kv.w));
        mo[k] = 0.f;
        ko[k] = 0.f;
        rev_finish<MODE>(yo[k], f4(lv, k), f4(mv, k), mb != 0, w, cw, kbn != nullptr, lo[k],
                         mo[k], ko[k]);
      }
      *reinterpret_cast<float4*>(y_or_lam + j0) = make_float4(lo[0], lo[1], lo[2], lo[3]);
      if (MODE == 1 && kbn) {
        *reinterpret_cast<float4*>(mu + j0) = make_float4(mo[0], mo[1], mo[2], mo[3]);
        *reinterpret_cast<float4*>(kbn + j0) = make_float4(ko[0], ko[1], ko[2], ko[3]);
      }
      if (MODE == 2 || MODE == 4)
        *reinterpret_cast<float4*>(kbn + j0) = make_float4(ko[0], ko[1], ko[2], ko[3]);
      return;
    }
#pragma unroll 1
    for (int k = 0; k < kRevVec && c0 + k < P; ++k)
      rev_one<DIR, MODE>(t, qx, qz, j0 + k, c0 + k < nx, r, c0 + k, P, rows, nx, y_or_lam, mask,
                         kbn, mu, w, cw);
    return;
  }
  const long long run = (long long)gridDim.x * kRevBlock * kRevVec;
  for (long long j = tail0 + (long long)blockIdx.y * run +
                     (long long)(blockIdx.x * kRevBlock + threadIdx.x) * kRevVec;
       j < L.len; j += (long long)gridDim.y * run) {
#pragma unroll 1
    for (int k = 0; k < kRevVec && j + k < L.len; ++k)
      rev_one<DIR, MODE>(t, qx, qz, j + k, false, 0, 0, P, 0, nx, y_or_lam, mask, kbn, mu, w, cw);
  }
}

// The CSR part of L^T x on the rows that have entries, kLanes threads per row:
// t[nzrow[r]] = sum over row r.
__global__ void k_rows_csr(const int* __restrict__ nzrow, const long long* __restrict__ rowptr,
                           const int* __restrict__ col, const float* __restrict__ val,
                           const float* __restrict__ x, long long nrows, float* t) {
  const long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / kLanes;
  const int lane = threadIdx.x % kLanes;
  if (r >= nrows) return;  // whole groups leave together
  const int j = nzrow[r];
  const float s = row_dot(rowptr, col, val, x, j, lane);
  if (lane == 0) t[j] = s;
}

__global__ void k_flag_rows(const long long* __restrict__ rowptr, long long len,
                            unsigned long long* flag) {
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j < len) flag[j] = rowptr[j + 1] > rowptr[j] ? 1ull : 0ull;
}

__global__ void k_list_rows(const long long* __restrict__ rowptr, const long long* __restrict__ pos,
                            long long len, int* nzrow) {
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j < len && rowptr[j + 1] > rowptr[j]) nzrow[pos[j]] = int(j);
}

__global__ void k_random(float* x, long long n, unsigned seed) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    unsigned h = unsigned(i) * 2654435761u ^ seed;
    h ^= h >> 15; h *= 2246822519u; h ^= h >> 13; h *= 3266489917u; h ^= h >> 16;
    x[i] = float(h) * (2.0f / 4294967296.0f) - 1.0f;
  }
}

unsigned grid_for(long long n, int block) {
  const long long b = (n + block - 1) / block;
  return unsigned(b < 148LL * 64 ? b : 148LL * 64);
}

}  // namespace

cudaError_t set_lattice(float* set, const SetLayout& L, int a, int cz, int cx, float v,
                        cudaStream_t st) {
  if (L.rows[a] <= 0) return cudaSuccess;
  k_set_lattice<<<dim3((L.ncols[a] + kBlock - 1) / kBlock, L.rows[a]), kBlock, 0, st>>>(set, L, a, cz,
                                                                                       cx, v);
  return cudaGetLastError();
}

cudaError_t fill(float* set, long long n, float v, cudaStream_t st) {
  k_fill<<<grid_for(n, kBlock), kBlock, 0, st>>>(set, n, v);
  return cudaGetLastError();
}

cudaError_t make_mask(const float* out, uint8_t* mask, long long n, cudaStream_t st) {
  k_mask<<<grid_for(n, kBlock), kBlock, 0, st>>>(out, mask, n);
  return cudaGetLastError();
}

cudaError_t extract(const float* out, const SetLayout& L, int a, int cz, int cx, float scale,
                    unsigned long long* count, const long long* rowptr, int* cursor, int* col,
                    float* val, int* err, cudaStream_t st) {
  k_extract<<<grid_for(L.len, kBlock), kBlock, 0, st>>>(out, L, a, cz, cx, scale, count, rowptr,
                                                        cursor, col, val, err);
  return cudaGetLastError();
}

cudaError_t scan(const unsigned long long* count, long long* rowptr, long long len, void** tmp,
                 size_t* tmp_bytes, cudaStream_t st) {
  size_t need = 0;
  auto* out = reinterpret_cast<unsigned long long*>(rowptr);
  cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, need, count, out, len + 1, st);
  if (e != cudaSuccess) return e;
  if (need > *tmp_bytes) {
    if (*tmp) cudaFree(*tmp);
    *tmp = nullptr;
    if ((e = cudaMalloc(tmp, need)) != cudaSuccess) return e;
    *tmp_bytes = need;
  }
  return cub::DeviceScan::ExclusiveSum(*tmp, need, count, out, len + 1, st);
}

cudaError_t sort_rows(const CsrT& A, long long len, cudaStream_t st) {
  k_sort_rows<<<unsigned((len + kBlock - 1) / kBlock), kBlock, 0, st>>>(A.rowptr, A.col, A.val, len);
  return cudaGetLastError();
}

cudaError_t drop_interior(const CsrT& full, const SetLayout& L, CsrT* rest,
                          unsigned long long* count, void** tmp, size_t* tmp_bytes, cudaStream_t st) {
  const unsigned g = unsigned((L.len + kBlock - 1) / kBlock);
  k_drop_count<<<g, kBlock, 0, st>>>(full.rowptr, full.col, L, count);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(count + L.len, 0, sizeof(unsigned long long), st)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&rest->rowptr, size_t(L.len + 1) * sizeof(long long))) != cudaSuccess) return e;
  if ((e = scan(count, rest->rowptr, L.len, tmp, tmp_bytes, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(&rest->nnz, rest->rowptr + L.len, sizeof(long long),
                           cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&rest->col, size_t(std::max<long long>(rest->nnz, 1)) * sizeof(int))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&rest->val, size_t(std::max<long long>(rest->nnz, 1)) * sizeof(float))) != cudaSuccess) return e;
  k_drop_fill<<<g, kBlock, 0, st>>>(full.rowptr, full.col, full.val, L, rest->rowptr, rest->col, rest->val);
  return cudaGetLastError();
}

cudaError_t list_rows(HybridT* H, const SetLayout& L, unsigned long long* flag, void** tmp,
                      size_t* tmp_bytes, cudaStream_t st) {
  const unsigned g = unsigned((L.len + kBlock - 1) / kBlock);
  k_flag_rows<<<g, kBlock, 0, st>>>(H->rest.rowptr, L.len, flag);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(flag + L.len, 0, sizeof(unsigned long long), st)) != cudaSuccess) return e;
  long long* pos = nullptr;
  if ((e = cudaMalloc(&pos, size_t(L.len + 1) * sizeof(long long))) != cudaSuccess) return e;
  e = scan(flag, pos, L.len, tmp, tmp_bytes, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&H->nrows, pos + L.len, sizeof(long long), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaMalloc(&H->nzrow, size_t(std::max<long long>(H->nrows, 1)) * sizeof(int));
  if (e == cudaSuccess) {
    k_list_rows<<<g, kBlock, 0, st>>>(H->rest.rowptr, pos, L.len, H->nzrow);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMalloc(&H->t, size_t(L.len) * sizeof(float));
  if (e == cudaSuccess) e = cudaMemsetAsync(H->t, 0, size_t(L.len) * sizeof(float), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(pos);
  return e;
}

cudaError_t random_fill(float* x, long long n, unsigned seed, cudaStream_t st) {
  k_random<<<grid_for(n, kBlock), kBlock, 0, st>>>(x, n, seed);
  return cudaGetLastError();
}

template <int DIR, int MODE>
static cudaError_t hybrid_t(const HybridT& H, const Coef& C, const SetLayout& L, const float* kb,
                            float* out, const uint8_t* mask, float* kbn, float* mu, float w,
                            float c, bool q_ready, cudaStream_t st) {
  if (!q_ready) {
    const dim3 gq(unsigned((L.nx + 127) / 128), unsigned(L.nzf + L.nzs));
    if (L.cpml) k_qfields<true><<<gq, 128, 0, st>>>(C, L, kb, H.qx, H.qz, H.t);
    else k_qfields<false><<<gq, 128, 0, st>>>(C, L, kb, H.qx, H.qz, H.t);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (H.nrows > 0 && !q_ready) {  // else formed by prepare()
    k_rows_csr<<<unsigned((H.nrows * kLanes + kBlock - 1) / kBlock), kBlock, 0, st>>>(
        H.nzrow, H.rest.rowptr, H.rest.col, H.rest.val, kb, H.nrows, H.t);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  // the main arrays are the fluid block [3][nz_f][P] at 0 and the solid block
  // [5][nz_s][P] at off[3]; the rest of the set follows the solid block
  const long long tail0 = L.off[3] + 5LL * L.nzs * L.pitch[3];
  const int gx = (L.pitch[0] + kRevBlock * kRevVec - 1) / (kRevBlock * kRevVec);
  const int gy = std::max(L.nzf, L.nzs);
  bool ok = L.off[0] == 0 && L.off[3] >= 3LL * L.nzf * L.pitch[0] && tail0 <= L.len && gy <= 65535 &&
            L.pitch[0] % 32 == 0 && L.off[3] % 32 == 0 && tail0 % kRevVec == 0;
  for (int a = 0; a < 8; ++a)
    ok = ok && L.pitch[a] == L.pitch[0] &&
         L.off[a] == (a < 3 ? (long long)a * L.nzf * L.pitch[0]
                            : L.off[3] + (long long)(a - 3) * L.nzs * L.pitch[0]);
  if (!ok) return cudaErrorInvalidValue;
  k_reverse_h<DIR, MODE><<<dim3(unsigned(gx), unsigned(gy), 9u), kRevBlock, 0, st>>>(
      H.t, H.qx, H.qz, L, tail0, out, mask, kbn, mu, w, c);
  return cudaGetLastError();
}

template <int MODE>
static cudaError_t hybrid_dir(const HybridT& H, const Coef& C, const SetLayout& L, int dir,
                              const float* kb, float* out, const uint8_t* mask, float* kbn,
                              float* mu, float w, float c, bool q_ready, cudaStream_t st) {
  return dir == kDirF ? hybrid_t<kDirF, MODE>(H, C, L, kb, out, mask, kbn, mu, w, c, q_ready, st)
                      : hybrid_t<kDirB, MODE>(H, C, L, kb, out, mask, kbn, mu, w, c, q_ready, st);
}

cudaError_t prepare(const HybridT& H, const Coef& C, const SetLayout& L, const float* kb,
                    cudaStream_t st) {
  const unsigned gx = unsigned((L.nx + 127) / 128);
  const long long per_row = (long long)gx * 128;
  const long long ycsr = H.nrows > 0 ? (H.nrows * kLanes + per_row - 1) / per_row : 0;
  const long long gy = L.nzf + L.nzs + ycsr;
  if (gy > 65535) return cudaErrorInvalidValue;
  const dim3 grid(gx, unsigned(gy));
  if (L.cpml)
    k_prepare<true><<<grid, 128, 0, st>>>(C, L, kb, H.qx, H.qz, H.t, H.nzrow, H.rest.rowptr,
                                          H.rest.col, H.rest.val, H.nrows);
  else
    k_prepare<false><<<grid, 128, 0, st>>>(C, L, kb, H.qx, H.qz, H.t, H.nzrow, H.rest.rowptr,
                                           H.rest.col, H.rest.val, H.nrows);
  return cudaGetLastError();
}

cudaError_t reverse_stage(const HybridT& H, const Coef& C, const SetLayout& L, int dir,
                          const float* kb, float* lam, const uint8_t* mask, bool mask_lam,
                          float* kbn, float* mu, float w, float c, bool q_ready, bool lam_from_mu,
                          cudaStream_t st) {
  if (!mask_lam) return hybrid_dir<1>(H, C, L, dir, kb, lam, mask, kbn, mu, w, c, q_ready, st);
  if (lam_from_mu) {
    if (!kbn) return cudaErrorInvalidValue;
    return hybrid_dir<4>(H, C, L, dir, kb, lam, mask, kbn, mu, w, c, q_ready, st);
  }
  if (kbn) return hybrid_dir<2>(H, C, L, dir, kb, lam, mask, kbn, mu, w, c, q_ready, st);
  return hybrid_dir<3>(H, C, L, dir, kb, lam, mask, kbn, mu, w, c, q_ready, st);
}

cudaError_t apply_t(const HybridT& H, const Coef& C, const SetLayout& L, int dir, const float* x,
                    float* y, cudaStream_t st) {
  if (H.qx) return hybrid_dir<0>(H, C, L, dir, x, y, nullptr, nullptr, nullptr, 0.f, 0.f, false, st);
  const unsigned grid = unsigned((L.len * kLanes + kBlock - 1) / kBlock);
  k_apply_t<<<grid, kBlock, 0, st>>>(H.rest.rowptr, H.rest.col, H.rest.val, x, y, L.len);
  return cudaGetLastError();
}

cudaError_t step_start(const float* lam, const SetLayout& L, const Coef& C, const float* res,
                       float* mu, float* kb, const uint8_t* mask, float c, cudaStream_t st) {
  if (L.nx < 7) return cudaSuccess;  // no interface columns 3..nx-4
  // the filter taps (src/elements.cu:30-33), as the forward finish kernel uses them
  const W7 w7{{1.1e-13f, 1.678e-06f, 0.03419f, 0.93163f, 0.03419f, 1.678e-06f, 1.1e-13f}};
  const unsigned blocks = unsigned((L.nx - 6 + kStartCols - 1) / kStartCols);
  k_step_start<<<blocks, dim3(kStartThreads, 8), 0, st>>>(lam, L, C.nrm, w7, res, mu, kb, mask, c);
  return cudaGetLastError();
}

template <int DIR, bool CPML>
static cudaError_t gradient_t(const Coef& C, const SetLayout& L, const Fields& Y, const Fields& KB,
                              const float* kb, float* qx, float* qz, const Grad& G, cudaStream_t st) {
  const int rows = 1 + (C.nzf - 4) + (C.nzs - 4);
  const unsigned gx = unsigned((C.nx + 127) / 128);
  k_grad_cells<DIR, CPML><<<dim3(gx, unsigned(rows)), 128, 0, st>>>(C, L, Y, KB, kb, qx, qz, G);
  return cudaGetLastError();
}

cudaError_t gradient(const Coef& C, const SetLayout& L, const Fields& Y, const float* kb,
                     double* const* g, int dir, HybridT* H, cudaStream_t st) {
  const Grad G{g[0], g[1], g[2], g[3], g[4], g[5], g[6]};
  Fields KB;
  float* p[kSetArrays];
  for (int a = 0; a < kSetArrays; ++a) p[a] = const_cast<float*>(kb) + L.off[a];
  KB.fvx = p[0]; KB.fvz = p[1]; KB.fp = p[2];
  KB.svx = p[3]; KB.svz = p[4]; KB.ssx = p[5]; KB.ssz = p[6]; KB.ssxz = p[7];
  for (int q = 0; q < 4; ++q) {
    KB.fx[q] = p[8 + q]; KB.sx[q] = p[12 + q]; KB.sz[q] = p[16 + q]; KB.fz[q] = p[20 + q];
  }
  float* qx = H ? H->qx : nullptr;
  float* qz = H ? H->qz : nullptr;
  if (C.cpml)
    return dir == kDirF ? gradient_t<kDirF, true>(C, L, Y, KB, kb, qx, qz, G, st)
                        : gradient_t<kDirB, true>(C, L, Y, KB, kb, qx, qz, G, st);
  return dir == kDirF ? gradient_t<kDirF, false>(C, L, Y, KB, kb, qx, qz, G, st)
                      : gradient_t<kDirB, false>(C, L, Y, KB, kb, qx, qz, G, st);
}

}  // namespace adj
}  // namespace mfdm
