// Phase-shift dispersion imaging of a receiver gather on the GPU (the
// reference's tools/test.py:50-98, `dispersion_imaging`).
//
// For a gather g[t][x] (nt samples of ntr traces at signed offsets x_r) with
// sampling rate fs:
//   S[k][r] = sum_t g[t][r] exp(-2 pi i k t / nt),   k = 0 .. nt/2   (rfft)
//   P[k][r] = conj(S[k][r]) / |S[k][r]|               (0 where |S| = 0)
//   A[k][j] = | sum_r P[k][r] exp(-i w_k x_r / c_j) | / ntr,
// w_k = 2 pi k fs / nt, c_j = c_min + j dc for c_j <= c_max + dc / 2.
// Two kernels, both accumulating in FP64 like the reference's numpy code:
// a direct DFT whose twiddles come from an exact table of nt roots of unity
// (index k t mod nt, in shared memory when it fits), then one thread per
// (frequency, velocity) stacking the phase-shifted traces. The gather is a few
// MB, so this is a compute pass (about nt^2 ntr / 2 + nf nc ntr complex
// multiply-adds), not an HBM-bound one.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/mfdm.h"
#include "mfdm_kernels.h"

namespace {

constexpr int kMaxTableSmem = 4096;  // roots of unity held in shared memory (64 KB of double2)

// S and P: thread per (trace r, frequency k); block = 128 traces of one k-tile.
__global__ void spectrum_kernel(const float* __restrict__ g, int nt, int ntr, int nf,
                                const double2* __restrict__ roots, double2* __restrict__ P) {
  extern __shared__ double2 tab[];
  const bool in_smem = nt <= kMaxTableSmem;
  if (in_smem)
    for (int m = threadIdx.x; m < nt; m += blockDim.x) tab[m] = roots[m];
  __syncthreads();
  const double2* w = in_smem ? tab : roots;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (r >= ntr || k >= nf) return;
  double re = 0.0, im = 0.0;
  int m = 0;  // k t mod nt, advanced by k each step
  for (int t = 0; t < nt; ++t) {
    const double v = double(__ldg(g + size_t(t) * ntr + r));
    const double2 e = w[m];
    re = fma(v, e.x, re);
    im = fma(v, e.y, im);
    m += k;
    if (m >= nt) m -= nt;
  }
  const double mag = sqrt(re * re + im * im);
  P[size_t(k) * ntr + r] = mag > 0.0 ? make_double2(re / mag, -im / mag) : make_double2(0.0, 0.0);
}

// A: thread per (velocity j, frequency k).
__global__ void image_kernel(const double2* __restrict__ P, const double* __restrict__ x, int ntr,
                             int nf, int nc, double dw, double c_min, double dc,
                             float* __restrict__ A) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (j >= nc || k >= nf) return;
  const double s = (double(k) * dw) / (c_min + double(j) * dc);  // w_k / c_j
  double re = 0.0, im = 0.0;
  for (int r = 0; r < ntr; ++r) {
    double sn, cs;
    sincos(-s * __ldg(x + r), &sn, &cs);
    const double2 p = P[size_t(k) * ntr + r];
    re += p.x * cs - p.y * sn;
    im += p.x * sn + p.y * cs;
  }
  A[size_t(k) * nc + j] = float(sqrt(re * re + im * im) / double(ntr));
}

int err(int code, const char* msg) { return mfdm::set_error(code, msg); }

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

extern "C" int mfdm_dispersion_velocities(double c_min, double c_max, double dc) {
  if (!(c_min > 0.0) || !(c_max >= c_min) || !(dc > 0.0) || !std::isfinite(c_max)) return 0;
  // numpy.arange(c_min, c_max + dc / 2, dc): ceil((stop - start) / step) values
  return int(std::ceil((c_max + dc / 2.0 - c_min) / dc));
}

extern "C" int mfdm_dispersion_image(const float* gather, int nt, int ntr, const double* offsets,
                                     double fs, double c_min, double c_max, double dc,
                                     float* amplitude, int device) {
  if (!gather || !offsets || !amplitude) return err(MFDM_ERR_ARG, "null argument");
  if (nt < 2 || ntr < 1) return err(MFDM_ERR_ARG, "need at least two samples and one trace");
  if (!(fs > 0.0) || !std::isfinite(fs)) return err(MFDM_ERR_ARG, "fs must be a positive finite value");
  const int nc = mfdm_dispersion_velocities(c_min, c_max, dc);
  if (nc <= 0) return err(MFDM_ERR_ARG, "velocities must satisfy 0 < c_min <= c_max and dc > 0");
  for (int r = 0; r < ntr; ++r)
    if (!std::isfinite(offsets[r])) return err(MFDM_ERR_ARG, "all offsets must be finite");
  const int nf = nt / 2 + 1;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return err(MFDM_ERR_ARG, "no such CUDA device");
  int prev = 0;
  cudaGetDevice(&prev);
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev};
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return err(MFDM_ERR_CUDA, cudaGetErrorString(e));
  // exact roots of unity exp(-2 pi i m / nt) in FP64, m = 0 .. nt-1
  std::vector<double2> roots(static_cast<size_t>(nt));
  for (int m = 0; m < nt; ++m) {
    const double a = -2.0 * M_PI * double(m) / double(nt);
    roots[size_t(m)] = make_double2(std::cos(a), std::sin(a));
  }
  DevBuf dg, dr, dx, dP, dA;
  const size_t gb = size_t(nt) * ntr * sizeof(float), rb = size_t(nt) * sizeof(double2),
               xb = size_t(ntr) * sizeof(double), pb = size_t(nf) * ntr * sizeof(double2),
               ab = size_t(nf) * nc * sizeof(float);
  if ((e = cudaMalloc(&dg.p, gb)) != cudaSuccess || (e = cudaMalloc(&dr.p, rb)) != cudaSuccess ||
      (e = cudaMalloc(&dx.p, xb)) != cudaSuccess || (e = cudaMalloc(&dP.p, pb)) != cudaSuccess ||
      (e = cudaMalloc(&dA.p, ab)) != cudaSuccess)
    return err(MFDM_ERR_NOMEM, cudaGetErrorString(e));
  if ((e = cudaMemcpy(dg.p, gather, gb, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(dr.p, roots.data(), rb, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(dx.p, offsets, xb, cudaMemcpyHostToDevice)) != cudaSuccess)
    return err(MFDM_ERR_CUDA, cudaGetErrorString(e));
  const size_t smem = nt <= kMaxTableSmem ? rb : 0;
  if (smem > 48 * 1024 &&
      (e = cudaFuncSetAttribute(spectrum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(smem))) != cudaSuccess)
    return err(MFDM_ERR_CUDA, cudaGetErrorString(e));
  spectrum_kernel<<<dim3(unsigned((ntr + 127) / 128), unsigned(nf)), 128, smem>>>(
      static_cast<const float*>(dg.p), nt, ntr, nf, static_cast<const double2*>(dr.p),
      static_cast<double2*>(dP.p));
  const double dw = 2.0 * M_PI * fs / double(nt);
  image_kernel<<<dim3(unsigned((nc + 127) / 128), unsigned(nf)), 128>>>(
      static_cast<const double2*>(dP.p), static_cast<const double*>(dx.p), ntr, nf, nc, dw, c_min,
      dc, static_cast<float*>(dA.p));
  if ((e = cudaGetLastError()) != cudaSuccess) return err(MFDM_ERR_CUDA, cudaGetErrorString(e));
  if ((e = cudaMemcpy(amplitude, dA.p, ab, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return err(MFDM_ERR_CUDA, cudaGetErrorString(e));
  return MFDM_OK;
}
