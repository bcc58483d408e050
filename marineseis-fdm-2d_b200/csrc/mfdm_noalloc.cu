// mfdm_step_noalloc: RK4 steps that allocate no memory.
//
// Some callers cannot allocate: a process that sets a fixed device-memory
// budget at start-up, code that runs where cudaMalloc is not allowed or would
// stall (a latency-critical loop, a host thread that must not synchronise the
// device through the allocator), or a framework whose own pool owns every
// byte of the GPU. Such a caller already holds the model and the wavefield in
// device memory; this entry point steps them with the library's kernels and
// keeps everything else it needs - the coefficient blocks in the kernels'
// layout, the RK stage buffers and accumulator, the ADE memory, the PML and
// source tables - in one file-scope device array of kNoAllocBytes. Every GPU
// that loads the library holds that array until the process exits.
//
// Calls share the array: calls that overlap on the GPU (two streams, two host
// threads) race and corrupt each other. The ADE memory in the array carries
// from one call to the next, so a run must start with it == 0 (which clears
// it) and continue with consecutive time indices on one model at a time.
// The Ricker and PML values come from the same host functions as the handle
// path's (mfdm::ricker_ref, mfdm::pml_cell), so both entry points step with
// bit-identical tables. The first call on a device caches the array's address
// and configures the kernels there; after cudaDeviceReset of that device the
// cache is stale, so a process that resets a device must not call this entry
// point on it again.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/mfdm.h"
#include "mfdm_kernels.h"

namespace {

constexpr size_t kNoAllocBytes = size_t(MFDM_NOALLOC_MAX_BYTES);
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct DeviceSlot {
  bool ready = false;
  unsigned char* base = nullptr;  // device address of g_noalloc_scratch on this device
};
DeviceSlot g_slots[kMaxDevices];
std::mutex g_setup_mutex;

// 5x5 source weights (src/elements.cu:34-40) and the interface filter (src/elements.cu:30-33).
const float kSrcW[25] = {0.0030f, 0.0133f, 0.0219f, 0.0133f, 0.0030f, 0.0133f, 0.0596f,
                         0.0983f, 0.0596f, 0.0133f, 0.0219f, 0.0983f, 0.1621f, 0.0983f,
                         0.0219f, 0.0133f, 0.0596f, 0.0983f, 0.0596f, 0.0133f, 0.0030f,
                         0.0133f, 0.0219f, 0.0133f, 0.0030f};
const float kW7[7] = {1.1e-13f, 1.678e-06f, 0.03419f, 0.93163f, 0.03419f, 1.678e-06f, 1.1e-13f};

int err(int code, const char* msg) { return mfdm::set_error(code, msg); }

#define NA_CU(call)                                                                  \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) return err(MFDM_ERR_CUDA, cudaGetErrorString(e_));        \
  } while (0)

// The first call on a device resolves the array's device address (host code
// cannot use the symbol itself) and configures the kernels on that device.
int setup_device(unsigned char** base) {
  int dev = -1;
  NA_CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return err(MFDM_ERR_ARG, "device index too large");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSlot& s = g_slots[dev];
  if (!s.ready) {
    void* p = nullptr;
    NA_CU(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (!p) return err(MFDM_ERR_CUDA, "no device address for the static scratch array");
    NA_CU(mfdm::configure_device());
    NA_CU(mfdm::upload_constants(kSrcW, kW7));
    s.base = static_cast<unsigned char*>(p);
    s.ready = true;
  }
  *base = s.base;
  return MFDM_OK;
}

// Rows of the Ricker table kept in the array: a call of more steps runs them
// in chunks of this many, refilling the table between chunks.
constexpr int kAmpSteps = 1024;
// Host staging of the tables: PML factors in pieces of this many cells.
constexpr int kPmlChunk = 256;

// Interface unit normals in FP64 from the metric on the device, with the host
// path's operations and rounding (no contraction into fused multiply-adds).
__global__ void normals_kernel(int nx, int nzf, int P, const float* zex, const float* zez,
                               float2* nrm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx) return;
  const size_t g = size_t(nzf - 1) * P + i;
  const double a = zex[g], b = zez[g];
  const double s = __dsqrt_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
  nrm[i] = s > 0 ? make_float2(float(__ddiv_rn(a, s)), float(__ddiv_rn(b, s)))
                 : make_float2(0.f, 1.f);
}

// Density slots hold 1/rho in the kernels' coefficient blocks (see mfdm_device.cuh).
__global__ void reciprocal_kernel(float* a, size_t n) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) a[i] = float(1.0 / double(a[i]));
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

}  // namespace

extern "C" int mfdm_step_noalloc(const mfdm_device_model* dm, int it, int nsteps, void* stream) {
  if (!dm) return err(MFDM_ERR_ARG, "null model");
  const int nx = dm->nx, nzf = dm->nz_f, nzs = dm->nz_s, npd = dm->npd;
  if (nx < 8 || nzf < 8 || nzs < 8) return err(MFDM_ERR_ARG, "grid too small: need nx, nz_f, nz_s >= 8");
  if (npd < 0 || 2 * npd > nx - 6 || npd > nzs) return err(MFDM_ERR_ARG, "PML width npd does not fit the grid");
  if (it < 0 || nsteps < 0) return err(MFDM_ERR_ARG, "negative time index or step count");
  if (!(dm->dt > 0.f) || !(dm->fpeak > 0.f)) return err(MFDM_ERR_ARG, "dt and fpeak must be > 0");
  if (dm->src_x >= 0 && (dm->src_x >= nx || dm->src_z < 0 || dm->src_z >= nzf))
    return err(MFDM_ERR_ARG, "source outside the fluid grid (src_x < 0 means no source)");
  const float* ins[12] = {dm->K, dm->rho_f, dm->C11, dm->C13, dm->C33, dm->C55,
                          dm->rho_s, dm->J, dm->xi_x, dm->xi_z, dm->ze_x, dm->ze_z};
  float* state[8] = {dm->vx_f, dm->vz_f, dm->p_f, dm->vx_s, dm->vz_s, dm->sx_s, dm->sz_s, dm->sxz_s};
  for (const float* p : ins)
    if (!p) return err(MFDM_ERR_ARG, "null model array");
  for (const float* p : state)
    if (!p) return err(MFDM_ERR_ARG, "null state array");

  // Layout of the scratch array (the same blocks an open handle allocates).
  const int nz = nzf + nzs - 1;
  const int P = round_up(nx > mfdm::kStageSW ? nx : mfdm::kStageSW, 32);
  const int Ps = round_up(2 * npd > 1 ? 2 * npd : 1, 4), npdr = npd > 1 ? npd : 1;
  size_t off = 0;
  auto take = [&](size_t nfloats) {
    const size_t o = off;
    off += (nfloats * sizeof(float) + 255) / 256 * 256;
    return o;
  };
  const size_t nf = size_t(nzf) * P, ns = size_t(nzs) * P, ng = size_t(nz) * P;
  const size_t o_fco = take(6 * nf), o_sco = take(9 * ns);
  size_t o_met[5];
  for (int q = 0; q < 5; ++q) o_met[q] = take(ng);
  const size_t o_pmlx = take(size_t(nx) * 4), o_pmlz = take(size_t(nzs) * 4),
               o_nrm = take(size_t(nx) * 2), o_ipre = take(size_t(8) * P), o_misc = take(64),
               o_amp = take(size_t(kAmpSteps) * 4);
  size_t o_fb[4], o_sb[4], o_ade[4][12];
  for (int s = 0; s < 4; ++s) {
    o_fb[s] = take(3 * nf);
    o_sb[s] = take(5 * ns);
  }
  const size_t o_ade_begin = off;
  for (int s = 0; s < 4; ++s) {
    for (int q = 0; q < 4; ++q) o_ade[s][q] = take(size_t(nzf) * Ps);
    for (int q = 0; q < 4; ++q) o_ade[s][4 + q] = take(size_t(nzs) * Ps);
    for (int q = 0; q < 4; ++q) o_ade[s][8 + q] = take(size_t(npdr) * P);
  }
  if (off > kNoAllocBytes) {
    char msg[200];
    snprintf(msg, sizeof msg,
             "model needs %zu bytes of scratch (%d x (%d + %d) cells); the static limit of "
             "mfdm_step_noalloc is %zu bytes (MFDM_NOALLOC_MAX_BYTES)",
             off, nx, nzf, nzs, kNoAllocBytes);
    return err(MFDM_ERR_ARG, msg);
  }

  unsigned char* base = nullptr;
  int rc = setup_device(&base);
  if (rc != MFDM_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  auto F = [&](size_t o) { return reinterpret_cast<float*>(base + o); };

  // Clear the transient blocks and the four RK sets; the ADE memory only at a run's start.
  NA_CU(cudaMemsetAsync(base, 0, o_ade_begin, st));
  if (it == 0) NA_CU(cudaMemsetAsync(base + o_ade_begin, 0, off - o_ade_begin, st));

  auto copy_rows = [&](float* dst, const float* src, int row0, int rows) -> int {
    NA_CU(cudaMemcpy2DAsync(dst, size_t(P) * 4, src + size_t(row0) * nx, size_t(nx) * 4,
                            size_t(nx) * 4, size_t(rows), cudaMemcpyDeviceToDevice, st));
    return MFDM_OK;
  };
  float* fco = F(o_fco);
  float* sco = F(o_sco);
  // fluid block: xi_x, xi_z, ze_x, ze_z (global rows 0..nz_f-1), rho, K
  // solid block: xi_x, xi_z, ze_x, ze_z (global rows nz_f-1..nz-1), rho, C11, C13, C33, C55
  const float* met[4] = {dm->xi_x, dm->xi_z, dm->ze_x, dm->ze_z};
  for (int q = 0; q < 4; ++q) {
    if ((rc = copy_rows(fco + q * nf, met[q], 0, nzf)) != MFDM_OK) return rc;
    if ((rc = copy_rows(sco + q * ns, met[q], nzf - 1, nzs)) != MFDM_OK) return rc;
  }
  if ((rc = copy_rows(fco + 4 * nf, dm->rho_f, 0, nzf)) || (rc = copy_rows(fco + 5 * nf, dm->K, 0, nzf)) ||
      (rc = copy_rows(sco + 4 * ns, dm->rho_s, 0, nzs)) || (rc = copy_rows(sco + 5 * ns, dm->C11, 0, nzs)) ||
      (rc = copy_rows(sco + 6 * ns, dm->C13, 0, nzs)) || (rc = copy_rows(sco + 7 * ns, dm->C33, 0, nzs)) ||
      (rc = copy_rows(sco + 8 * ns, dm->C55, 0, nzs)))
    return rc;
#if MFDM_RCP_RHO
  // rows x pitch of each density slot; the padding columns become 1/0 = inf and are never read
  reciprocal_kernel<<<unsigned((nf + 255) / 256), 256, 0, st>>>(fco + 4 * nf, nf);
  reciprocal_kernel<<<unsigned((ns + 255) / 256), 256, 0, st>>>(sco + 4 * ns, ns);
  NA_CU(cudaGetLastError());
#endif
  const float* gmet[5] = {dm->J, dm->xi_x, dm->xi_z, dm->ze_x, dm->ze_z};
  for (int q = 0; q < 5; ++q)
    if ((rc = copy_rows(F(o_met[q]), gmet[q], 0, nz)) != MFDM_OK) return rc;

  // The wavefield in: the caller's arrays become set U.
  mfdm::Fields S[4] = {};
  for (int s = 0; s < 4; ++s) {
    float* fb = F(o_fb[s]);
    float* sb = F(o_sb[s]);
    S[s].fvx = fb; S[s].fvz = fb + nf; S[s].fp = fb + 2 * nf;
    S[s].svx = sb; S[s].svz = sb + ns; S[s].ssx = sb + 2 * ns; S[s].ssz = sb + 3 * ns;
    S[s].ssxz = sb + 4 * ns;
    for (int q = 0; q < 4; ++q) {
      S[s].fx[q] = F(o_ade[s][q]);
      S[s].sx[q] = F(o_ade[s][4 + q]);
      S[s].sz[q] = F(o_ade[s][8 + q]);
    }
  }
  float* const u_dst[8] = {S[0].fvx, S[0].fvz, S[0].fp, S[0].svx, S[0].svz, S[0].ssx, S[0].ssz, S[0].ssxz};
  for (int f = 0; f < 8; ++f)
    if ((rc = copy_rows(u_dst[f], state[f], 0, f < 3 ? nzf : nzs)) != MFDM_OK) return rc;

  // PML factors on the host (the handle path's function), in pieces through a
  // stack buffer: pageable copies return once the source is staged.
  {
    float4 buf[kPmlChunk];
    float4* const pml[2] = {reinterpret_cast<float4*>(F(o_pmlx)), reinterpret_cast<float4*>(F(o_pmlz))};
    const int len[2] = {nx, nzs};
    for (int a = 0; a < 2; ++a)
      for (int i0 = 0; i0 < len[a]; i0 += kPmlChunk) {
        const int n = len[a] - i0 < kPmlChunk ? len[a] - i0 : kPmlChunk;
        for (int i = 0; i < n; ++i)
          buf[i] = mfdm::pml_cell(dm->fpeak, dm->beta0, npd, dm->npow, dm->vp_max, dm->rc,
                                  dm->thickness, i0 + i, len[a], a == 0, true);
        NA_CU(cudaMemcpyAsync(pml[a] + i0, buf, size_t(n) * sizeof(float4), cudaMemcpyHostToDevice, st));
      }
  }
  normals_kernel<<<(nx + 255) / 256, 256, 0, st>>>(nx, nzf, P, F(o_met[3]), F(o_met[4]),
                                                   reinterpret_cast<float2*>(F(o_nrm)));
  NA_CU(cudaGetLastError());

  mfdm::Coef C{};
  C.nx = nx; C.nzf = nzf; C.nzs = nzs; C.P = P; C.npd = npd; C.Ps = Ps;
  C.rhof = fco + 4 * nf; C.K = fco + 5 * nf;
  C.rhos = sco + 4 * ns; C.C11 = sco + 5 * ns; C.C13 = sco + 6 * ns; C.C33 = sco + 7 * ns;
  C.C55 = sco + 8 * ns;
  C.J = F(o_met[0]); C.xix = F(o_met[1]); C.xiz = F(o_met[2]); C.zex = F(o_met[3]); C.zez = F(o_met[4]);
  C.pmlx = reinterpret_cast<const float4*>(F(o_pmlx));
  C.pmlz = reinterpret_cast<const float4*>(F(o_pmlz));
  C.nrm = reinterpret_cast<const float2*>(F(o_nrm));
  // Ricker table rows: time indices src_it0 .. src_it0 + src_steps - 1 (set per chunk below).
  C.src_amp = F(o_amp);
  C.srcx = dm->src_x;
  C.srcz = dm->src_z;
  const float dt = dm->dt;
  C.rk_c[0] = dt / 2; C.rk_c[1] = dt / 2; C.rk_c[2] = dt; C.rk_c[3] = dt / 6.0f;
  C.rk_w[0] = dt / 6; C.rk_w[1] = dt / 3; C.rk_w[2] = dt / 3;
  C.gap = 1;
  C.rec = nullptr;  // receivers: the caller reads its own state arrays
  C.rec_cap = 0;
  C.ipre = F(o_ipre);
  int* misc = reinterpret_cast<int*>(F(o_misc));
  C.step = misc;
  C.done = reinterpret_cast<unsigned*>(misc + 1);
  C.status = misc + 2;

  CUtensorMap fst[4], sst[4], fpw[4], spw[4], fcm, scm;
  for (int s = 0; s < 4; ++s) {
    // state maps: one shot (the kernels address the shot as a fourth coordinate)
    if ((rc = mfdm::encode_block_map(&fst[s], F(o_fb[s]), P, nzf, 3, mfdm::kStageSW, true, 1, 256)) ||
        (rc = mfdm::encode_block_map(&sst[s], F(o_sb[s]), P, nzs, 5, mfdm::kStageSW, true, 1, 256)) ||
        (rc = mfdm::encode_block_map(&fpw[s], F(o_fb[s]), P, nzf, 3, mfdm::kStageTX, false, 1, 256)) ||
        (rc = mfdm::encode_block_map(&spw[s], F(o_sb[s]), P, nzs, 5, mfdm::kStageTX, false, 1, 256)))
      return rc;
  }
  if ((rc = mfdm::encode_block_map(&fcm, fco, P, nzf, 6, mfdm::kStageTX, false)) ||
      (rc = mfdm::encode_block_map(&scm, sco, P, nzs, 9, mfdm::kStageTX, false)))
    return rc;

  NA_CU(mfdm::launch_set_step(C, it, st));
  const int in_set[4] = {0, 1, 2, 1}, out_set[4] = {1, 2, 1, 0};
  const float half = float(double(dt) * 0.5);
  for (int k0 = 0; k0 < nsteps; k0 += kAmpSteps) {
    const int nk = nsteps - k0 < kAmpSteps ? nsteps - k0 : kAmpSteps;
    // The chunk's Ricker values on the host with the handle path's function
    // (src/elements.cu:385-392, float time = it * dt), staged from the stack.
    // The copy is ordered after the previous chunk's kernels on this stream.
    {
      float amp[kAmpSteps * 4];
      for (int k = 0; k < nk; ++k) {
        const float t = float(it + k0 + k) * dt;
        amp[k * 4 + 0] = mfdm::ricker_ref(dm->fpeak, t);
        amp[k * 4 + 1] = mfdm::ricker_ref(dm->fpeak, t + half);
        amp[k * 4 + 2] = mfdm::ricker_ref(dm->fpeak, t + half);
        amp[k * 4 + 3] = mfdm::ricker_ref(dm->fpeak, t + dt);
      }
      NA_CU(cudaMemcpyAsync(F(o_amp), amp, size_t(nk) * 4 * sizeof(float), cudaMemcpyHostToDevice, st));
    }
    C.src_it0 = it + k0;
    C.src_steps = nk;
    for (int k = k0; k < k0 + nk; ++k) {
      const int d0 = ((it + k) & 1) ? mfdm::kDirB : mfdm::kDirF, d1 = 1 - d0;
      const int dir[4] = {d0, d1, d0, d1};
      for (int s = 0; s < 4; ++s) {
        mfdm::StageMaps maps;
        maps.fin = fst[in_set[s]];
        maps.sin = sst[in_set[s]];
        maps.fun = fpw[0];
        maps.sun = spw[0];
        maps.facc = fpw[3];
        maps.sacc = spw[3];
        maps.fcoef = fcm;
        maps.scoef = scm;
        NA_CU(mfdm::launch_stage(C, S[in_set[s]], S[out_set[s]], S[0], S[3], maps, s, dir[s], st));
      }
      NA_CU(mfdm::launch_finish(C, S[0], st));
    }
  }
  // The wavefield out.
  for (int f = 0; f < 8; ++f)
    NA_CU(cudaMemcpy2DAsync(state[f], size_t(nx) * 4, u_dst[f], size_t(P) * 4, size_t(nx) * 4,
                            size_t(f < 3 ? nzf : nzs), cudaMemcpyDeviceToDevice, st));
  int status = 0;
  NA_CU(cudaMemcpyAsync(&status, C.status, sizeof(int), cudaMemcpyDeviceToHost, st));
  NA_CU(cudaStreamSynchronize(st));
  if (status & 2)
    return err(MFDM_ERR_CUDA, "a stage kernel pipeline wait timed out; the state arrays are undefined");
  if (status & 1) return err(MFDM_ERR_NONFINITE, "non-finite values reached the interface rows");
  return MFDM_OK;
}
