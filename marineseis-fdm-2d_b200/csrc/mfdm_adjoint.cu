// sm_100a kernels of the adjoint-state backward (see mfdm_adjoint.h).
#include <cub/device/device_scan.cuh>

#include "mfdm_adjoint.h"

namespace mfdm {
namespace adj {
namespace {

constexpr int kLanes = 8;  // threads per CSR row in the transposed products
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
__device__ __forceinline__ float row_dot(const long long* __restrict__ rowptr,
                                         const int* __restrict__ col, const float* __restrict__ val,
                                         const float* __restrict__ x, long long row, int lane) {
  float s = 0.0f;
  const long long e = rowptr[row + 1];
  for (long long k = rowptr[row] + lane; k < e; k += kLanes) s = fmaf(val[k], __ldg(x + col[k]), s);
  const unsigned grp = 0xFFu << (threadIdx.x & 24);
#pragma unroll
  for (int o = kLanes / 2; o > 0; o >>= 1) s += __shfl_xor_sync(grp, s, o);
  return s;
}

template <bool MASK_LAM, bool NEXT>
__global__ void k_reverse(const long long* __restrict__ rowptr, const int* __restrict__ col,
                          const float* __restrict__ val, const float* __restrict__ kb, float* lam,
                          const uint8_t* __restrict__ mask, float* kbn, const float* __restrict__ mu,
                          float w, float c, long long len) {
  const long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / kLanes;
  const int lane = threadIdx.x % kLanes;
  if (row >= len) return;  // whole groups leave together
  const float y = row_dot(rowptr, col, val, kb, row, lane);
  if (lane == 0) {
    const float m = mask[row] ? 1.0f : 0.0f;
    lam[row] += MASK_LAM ? m * y : y;
    if (NEXT) kbn[row] = m * fmaf(c, y, w * mu[row]);
  }
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

// Receivers sample the filtered interface rows of columns 3..nx-4
// (elsewhere the record is 0 whatever the state).
__global__ void k_inject(float* lam, SetLayout L, const float* __restrict__ res) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  if (ix < 3 || ix > L.nx - 4) return;
  const int nx = L.nx;
  lam[L.off[3] + ix] += res[ix];
  lam[L.off[4] + ix] += res[nx + ix];
  lam[L.off[2] + (long long)(L.nzf - 1) * L.pitch[2] + ix] += res[2 * nx + ix];
}

struct W7 { float w[7]; };

__device__ __forceinline__ long long iface_index(const SetLayout& L, int f, int ix) {
  return f < 3 ? L.off[f] + (long long)(L.nzf - 1) * L.pitch[f] + ix : L.off[f] + ix;
}

// Transposed continuity average of column ix, divided by the column's tap sum:
// tmp[f][ix] = (A^T lam)_f / wsum(ix).
__global__ void k_filter_t_a(const float* lam, SetLayout L, const float2* __restrict__ nrm,
                             float* tmp, W7 w7) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = L.nx;
  if (ix < 3 || ix > nx - 4) return;
  float lv[8];
#pragma unroll
  for (int f = 0; f < 8; ++f) lv[f] = lam[iface_index(L, f, ix)];
  const int klo = max(-3, 3 - ix), khi = min(3, nx - 4 - ix);
  float wsum = 0.0f;
  for (int k = klo; k <= khi; ++k) wsum += w7.w[k + 3];
  const float2 n = __ldg(nrm + ix);
#pragma unroll
  for (int f = 0; f < 8; ++f) {
    float e[8], u[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) e[q] = q == f ? 1.0f : 0.0f;
    interface_average(n, e, u);
    float t = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q) t = fmaf(lv[q], u[q], t);
    tmp[f * nx + ix] = t / wsum;
  }
}

// Transposed smoothing: lam at interface cell (f, j) = sum_k w_k tmp[f][j - k].
__global__ void k_filter_t_b(float* lam, SetLayout L, const float* __restrict__ tmp, W7 w7) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = L.nx;
  if (j < 3 || j > nx - 4) return;
#pragma unroll
  for (int f = 0; f < 8; ++f) {
    float s = 0.0f;
#pragma unroll
    for (int k = -3; k <= 3; ++k) {
      const int i = j - k;
      if (i >= 3 && i <= nx - 4) s = fmaf(w7.w[k + 3], tmp[f * nx + i], s);
    }
    lam[iface_index(L, f, j)] = s;
  }
}

__global__ void k_start(const float* __restrict__ lam, float* mu, float* kb,
                        const uint8_t* __restrict__ mask, long long n, float c) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float l = lam[i];
    mu[i] = l;
    kb[i] = mask[i] ? c * l : 0.0f;
  }
}

// ---- material gradients ----------------------------------------------------------

struct Grad {
  double *K, *rf, *c11, *c13, *c33, *c55, *rs;
};

// Fluid rows 3..nz_f-2 then solid rows 1..nz_s-4 (blockIdx.y), columns 3..nx-4.
template <int DIR, bool CPML>
__global__ void __launch_bounds__(128) k_grad_cells(Coef C, Fields Y, Fields KB, Grad G) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = C.nx, P = C.P, nzf = C.nzf, nzs = C.nzs, npd = C.npd;
  if (ix < 3 || ix > nx - 4) return;
  const bool side = min(ix - 3, nx - 4 - ix) < npd;
  const int scol = side ? xstrip_col(ix, nx, npd) : 0;
  const int nfr = nzf - 4;
  const int row = blockIdx.y;
  if (row < nfr) {
    const int iz = 3 + row;
    const size_t g = (size_t)iz * P + ix;
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
    G.rf[g] += double(__ldg(KB.fvx + g)) * o.vx + double(__ldg(KB.fvz + g)) * o.vz;
    G.K[g] += double(__ldg(KB.fp + g)) * o.p;
    return;
  }
  const int iz = 1 + row - nfr;
  if (iz > nzs - 4) return;
  const size_t m = (size_t)iz * P + ix, g = m + (size_t)(nzf - 1) * P;
  const int zb0 = nzs - 3 - npd;
  const bool bottom = iz >= zb0;
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
  const SolidK o2 = solid_rhs<DIR, false, CPML>(C, A, iz, ix, side, bottom, xade, zade,
                                                SolidCoefs{xix, xiz, zex, zez, 0.f, 0.f, 1.f, 0.f, 0.f});
  G.c11[m] += ksx * o1.sx;
  G.c33[m] += ksz * o1.sz;
  G.c55[m] += ksxz * o1.sxz;
  G.rs[m] += kvx * o1.vx + kvz * o1.vz;
  G.c13[m] += ksx * o2.sx + ksz * o2.sz;
}

// Interface column ix: both media's RHS at the interface row, coupled, per coefficient.
template <int DIR, bool CPML>
__global__ void __launch_bounds__(128) k_grad_iface(Coef C, Fields Y, Fields KB, Grad G) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = C.nx, P = C.P, nzf = C.nzf, nzs = C.nzs, npd = C.npd;
  if (ix < 3 || ix > nx - 4) return;
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

cudaError_t reverse_stage(const CsrT& A, long long len, const float* kb, float* lam,
                          const uint8_t* mask, bool mask_lam, float* kbn, const float* mu, float w,
                          float c, cudaStream_t st) {
  const unsigned grid = unsigned((len * kLanes + kBlock - 1) / kBlock);
  if (mask_lam && kbn)
    k_reverse<true, true><<<grid, kBlock, 0, st>>>(A.rowptr, A.col, A.val, kb, lam, mask, kbn, mu, w, c, len);
  else if (mask_lam)
    k_reverse<true, false><<<grid, kBlock, 0, st>>>(A.rowptr, A.col, A.val, kb, lam, mask, kbn, mu, w, c, len);
  else if (kbn)
    k_reverse<false, true><<<grid, kBlock, 0, st>>>(A.rowptr, A.col, A.val, kb, lam, mask, kbn, mu, w, c, len);
  else
    k_reverse<false, false><<<grid, kBlock, 0, st>>>(A.rowptr, A.col, A.val, kb, lam, mask, kbn, mu, w, c, len);
  return cudaGetLastError();
}

cudaError_t apply_t(const CsrT& A, long long len, const float* x, float* y, cudaStream_t st) {
  const unsigned grid = unsigned((len * kLanes + kBlock - 1) / kBlock);
  k_apply_t<<<grid, kBlock, 0, st>>>(A.rowptr, A.col, A.val, x, y, len);
  return cudaGetLastError();
}

cudaError_t inject(float* lam, const SetLayout& L, const float* res, cudaStream_t st) {
  k_inject<<<(L.nx + kBlock - 1) / kBlock, kBlock, 0, st>>>(lam, L, res);
  return cudaGetLastError();
}

cudaError_t filter_t(float* lam, const SetLayout& L, const Coef& C, float* tmp, cudaStream_t st) {
  // the filter taps (src/elements.cu:30-33), as the forward finish kernel uses them
  const W7 w7{{1.1e-13f, 1.678e-06f, 0.03419f, 0.93163f, 0.03419f, 1.678e-06f, 1.1e-13f}};
  const unsigned g = unsigned((L.nx + kBlock - 1) / kBlock);
  k_filter_t_a<<<g, kBlock, 0, st>>>(lam, L, C.nrm, tmp, w7);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_filter_t_b<<<g, kBlock, 0, st>>>(lam, L, tmp, w7);
  return cudaGetLastError();
}

cudaError_t start(const float* lam, float* mu, float* kb, const uint8_t* mask, long long n, float c,
                  cudaStream_t st) {
  k_start<<<grid_for(n, kBlock), kBlock, 0, st>>>(lam, mu, kb, mask, n, c);
  return cudaGetLastError();
}

template <int DIR, bool CPML>
static cudaError_t gradient_t(const Coef& C, const Fields& Y, const Fields& KB, const Grad& G,
                              cudaStream_t st) {
  const int rows = (C.nzf - 4) + (C.nzs - 4);
  const unsigned gx = unsigned((C.nx + 127) / 128);
  k_grad_cells<DIR, CPML><<<dim3(gx, unsigned(rows)), 128, 0, st>>>(C, Y, KB, G);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_grad_iface<DIR, CPML><<<gx, 128, 0, st>>>(C, Y, KB, G);
  return cudaGetLastError();
}

cudaError_t gradient(const Coef& C, const Fields& Y, const Fields& KB, double* const* g, int dir,
                     cudaStream_t st) {
  const Grad G{g[0], g[1], g[2], g[3], g[4], g[5], g[6]};
  if (C.cpml)
    return dir == kDirF ? gradient_t<kDirF, true>(C, Y, KB, G, st) : gradient_t<kDirB, true>(C, Y, KB, G, st);
  return dir == kDirF ? gradient_t<kDirF, false>(C, Y, KB, G, st) : gradient_t<kDirB, false>(C, Y, KB, G, st);
}

}  // namespace adj
}  // namespace mfdm
