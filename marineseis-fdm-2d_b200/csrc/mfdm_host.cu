// Host side of libmfdm: the C ABI declared in include/mfdm.h.
//
// Replaces the reference's MemManager (src/elements.cu), the stream handshake
// and the launch sequence of PmlFs::FluidSolid::update_RK4
// (src/pml_fs_kernels.cu:533-868) and the drop-in CLI (src/main.cu). One
// non-blocking stream per handle; the time loop is captured once as a CUDA
// graph of kGraphSteps steps and replayed; receivers are sampled on the
// device into a buffer drained once per shot.
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <future>
#include <iomanip>
#include <iostream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mfdm.h"
#include "json_config.h"
#include "mfdm_adjoint.h"
#include "mfdm_kernels.h"
#include "mfdm_solid.h"

namespace fs = std::filesystem;
using mfdm::Coef;
using mfdm::Fields;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define MFDM_CU(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(e_ == cudaErrorMemoryAllocation ? MFDM_ERR_NOMEM : MFDM_ERR_CUDA,     \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                  \
  } while (0)

constexpr int kGraphSteps = 32;  // steps per captured graph (must be even)

// 5x5 source weights (src/elements.cu:34-40) and the interface filter (src/elements.cu:30-33).
const float kSrcW[25] = {0.0030f, 0.0133f, 0.0219f, 0.0133f, 0.0030f, 0.0133f, 0.0596f,
                         0.0983f, 0.0596f, 0.0133f, 0.0219f, 0.0983f, 0.1621f, 0.0983f,
                         0.0219f, 0.0133f, 0.0596f, 0.0983f, 0.0596f, 0.0133f, 0.0030f,
                         0.0133f, 0.0219f, 0.0133f, 0.0030f};
const float kW7[7] = {1.1e-13f, 1.678e-06f, 0.03419f, 0.93163f, 0.03419f, 1.678e-06f, 1.1e-13f};

struct HostModel {
  int nx = 0, nzf = 0, nzs = 0;
  float fpeak = 0.f, dt = 0.f;
  int nt = 0, snapshot = 1;
  int npd = 0, npow = 2;
  float thickness = 0.f, vp_max = 0.f, rc = 0.f, beta0 = 1.f;
  int bdy = 2;  // boundary type: 2 free surface on top (PANDF), 1 CFS-PML on all sides (CPML)
  std::vector<int> srcx, srcz;
  // host arrays, [rows][nx], when the model was read from files
  std::vector<float> K, rhof, C11, C13, C33, C55, rhos, J, xix, xiz, zex, zez;
  // The arrays the upload reads: the vectors above, or the caller's own memory
  // (mfdm_desc), which is then copied to the device directly, without a host copy.
  struct View {
    const float *K, *rhof, *C11, *C13, *C33, *C55, *rhos, *J, *xix, *xiz, *zex, *zez;
  } v{};
  void view_own() {
    v = {K.data(), rhof.data(), C11.data(), C13.data(), C33.data(), C55.data(),
         rhos.data(), J.data(), xix.data(), xiz.data(), zex.data(), zez.data()};
  }
};

int round_up(int v, int m) { return (v + m - 1) / m * m; }

}  // namespace

namespace mfdm {
// Ricker wavelet in the reference's host arithmetic (src/elements.cu:385-392):
// float time, T = 1.2 / fpeak, the phase product in double rounded to float.
float ricker_ref(float fpeak, float time) {
  const float T = float(1.2 / double(fpeak));
  const float t = time - T;
  if (t > T) return 0.0f;
  float temp = float(M_PI * double(fpeak) * double(t));
  temp *= temp;
  return (1 - 2 * temp) * expf(-temp);
}

// CFS-PML factors of cell i of an axis of n cells in FP64 (src/elements.cu:121-124,
// 824-873): d = d0 r^NPOW, beta = 1 + (beta0-1) r^2, alpha = alpha0 (1 - r),
// r = k/npd, k counted from the inner edge of the band of npd cells inside 3
// frozen cells (lo: the band at the low end, hi: at the high end). Stored as
// (d/beta, alpha + d/beta, 1/beta), the factors the reference derives inside
// every kernel.
float4 pml_cell(float fpeak, float beta0, int npd, int npow, float vp_max, float rc,
                float thickness, int i, int n, bool lo, bool hi) {
  const double alpha0 = 2.0 * M_PI * double(fpeak);
  const double d0 = -(npow + 1) * double(vp_max) * std::log(double(rc)) / (2.0 * double(thickness));
  int k = -1;
  if (lo && i >= 3 && i <= 2 + npd) k = 3 + npd - i;
  if (hi && i >= n - 3 - npd && i <= n - 4) k = i - (n - 4 - npd);
  double d = 0.0, be = 1.0, al = alpha0;
  if (k > 0) {
    const double r = double(k) / double(npd);
    d = d0 * std::pow(r, double(npow));
    be = 1.0 + (double(beta0) - 1.0) * r * r;
    al = alpha0 * (1.0 - r);
  }
  const double dpb = d / be;
  return make_float4(float(dpb), float(al + dpb), float(1.0 / be), 0.f);
}
}  // namespace mfdm

namespace {
using mfdm::ricker_ref;

// One shot of a handle: source cell and Ricker peak frequency, and the PML
// beta0 that goes with it (alpha0 = 2 pi fpeak follows the frequency).
struct ShotCfg {
  int x = -1, z = 0;
  float fpeak = 0.f, beta0 = 1.f;
};

}  // namespace

struct AdjointState;

struct mfdm_model {
  int device = 0;
  int nshots = 1;              // shots stepped together (1 for a plain handle)
  std::vector<ShotCfg> shots;  // per-shot source, frequency and PML beta0
  bool batch = false;          // opened with mfdm_open_batch
  size_t region = 0;           // bytes of one shot's state region
  int* d_srcpos = nullptr;     // per-shot source cells (batch handles)
  cudaStream_t stream = nullptr;
  HostModel cfg;  // scalars (arrays released after upload)
  int P = 0, Ps = 0, nz = 0, gap = 1;
  int isrc = 0;
  int host_step = 0;
  char* dmem = nullptr;
  size_t dbytes = 0;
  Fields S[4];  // U, stage A, stage B, accumulator
  Coef C{};
  float* d_src = nullptr;
  int src_steps = 0;
  float* d_rec = nullptr;
  int rec_cap = 0;
  cudaGraphExec_t graph = nullptr;
  unsigned gen = 0;  // bumped whenever captured launches go stale (groups recapture)
  // TMA descriptors: per RK set (U, A, B, acc) the stencil box and the
  // point-wise box of the fluid and solid blocks, and the coefficient blocks.
  CUtensorMap fst[4], sst[4], fpw[4], spw[4], fco, sco;
  float* fcoef = nullptr;  // [6][nz_f][P]: xi_x, xi_z, ze_x, ze_z, rho, K
  float* scoef = nullptr;  // [9][nz_s][P]: xi_x, xi_z, ze_x, ze_z, rho, C11, C13, C33, C55
  AdjointState* adj = nullptr;  // adjoint operators and buffers (mfdm_adjoint_*)
  long long adj_keep_budget = 0;  // mfdm_adjoint_set_memory
  int adj_inner = 0;              // mfdm_adjoint_set_inner: second checkpoint level (0: none)
};

// Device buffers of the adjoint (one plain handle): the transposed stage
// operators of both directions, the updated-cell mask, the adjoint sets, the
// material gradients, the checkpoints of the forward run and the stage inputs
// of one checkpoint segment.
struct AdjointState {
  mfdm::SetLayout L{};
  mfdm::HybridT H[2];      // transposed stage operators, F and B (shared Q buffers)
  uint8_t* mask = nullptr;
  float *lam = nullptr, *mu = nullptr, *kb[2] = {nullptr, nullptr};
  double* grad = nullptr;  // K, 1/rho_f [nz_f][P]; C11, C13, C33, C55, 1/rho_s [nz_s][P]
  bool grad_ready = false;  // grad holds a finished backward pass
  float* ckpt = nullptr;   // checkpoint sets
  size_t ckpt_sets = 0;
  float* seg = nullptr;    // 4 stage-input sets per step of one segment
  float* seg2 = nullptr;   // a second such buffer: the next segment is recomputed into it
  size_t seg_steps = 0;    // while this one is reversed (when the memory allows)
  float* keep = nullptr;   // stage inputs of the last `nkeep` segments, kept by the forward pass
  size_t keep_floats = 0;
  // TMA maps of every step slot's four stage-input sets (stencil boxes) and of
  // its first set as U^n (point-wise boxes), per buffer of slots (keep, seg,
  // seg2): kept and recomputed steps run their stages in place in the slots
  struct SlotMaps { CUtensorMap fst[4], sst[4], fun, sun; };
  struct SlotTable {
    const float* base = nullptr;
    std::vector<SlotMaps> maps;
  };
  SlotTable keep_tab, seg_tab[2];
  int nkeep = 0;
  float* res = nullptr;    // residual samples [ns][3][nx]
  float* inner = nullptr;  // second-level checkpoints of one segment
  size_t inner_sets = 0;
  size_t res_floats = 0;
  void* scan_tmp = nullptr;
  size_t scan_bytes = 0;
  bool built = false;
  // Streams of the backward steps: `hi` runs the transposed chain at the
  // highest priority, `side_g` the material-gradient accumulation at the
  // lowest, so its blocks take only the SMs the chain leaves idle.
  cudaStream_t hi = nullptr, side_g = nullptr;
  cudaEvent_t ev_kb = nullptr, ev_g[2] = {nullptr, nullptr};
  cudaEvent_t ev_enter = nullptr, ev_leave = nullptr;
  cudaEvent_t ev_seg[2] = {nullptr, nullptr};  // segment recomputed into seg / seg2
  cudaEvent_t ev_rev[2] = {nullptr, nullptr};  // last reverse reading seg / seg2 done
  int nsteps = -1, every = 0;  // the forward run a backward pass may follow
  double build_ms = 0.0;       // operator assembly time (host clock)
  ~AdjointState() {
    for (auto& h : H) {
      cudaFree(h.rest.rowptr);
      cudaFree(h.rest.col);
      cudaFree(h.rest.val);
      cudaFree(h.nzrow);
      cudaFree(h.t);
    }
    cudaFree(H[0].qx);
    cudaFree(H[0].qz);
    cudaFree(mask); cudaFree(lam); cudaFree(mu); cudaFree(kb[0]); cudaFree(kb[1]);
    cudaFree(grad); cudaFree(ckpt); cudaFree(seg); cudaFree(res); cudaFree(keep);
    cudaFree(inner);
    cudaFree(scan_tmp);
    if (ev_kb) cudaEventDestroy(ev_kb);
    if (ev_enter) cudaEventDestroy(ev_enter);
    if (ev_leave) cudaEventDestroy(ev_leave);
    for (cudaEvent_t e : ev_seg)
      if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ev_rev)
      if (e) cudaEventDestroy(e);
    cudaFree(seg2);
    if (hi) cudaStreamDestroy(hi);
    for (cudaEvent_t e : ev_g)
      if (e) cudaEventDestroy(e);
    if (side_g) cudaStreamDestroy(side_g);
  }
};

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int validate(const HostModel& h) {
  if (h.nx < 8 || h.nzf < 8 || h.nzs < 8)
    return fail(MFDM_ERR_ARG, "grid too small: need nx, nz_f, nz_s >= 8");
  if (h.npd < 0 || 2 * h.npd > h.nx - 6 || h.npd > h.nzs)
    return fail(MFDM_ERR_ARG, "PML width npd does not fit the grid");
  if (h.bdy == 1 && h.npd + 3 > h.nzf)
    return fail(MFDM_ERR_ARG, "the top PML band (rows 3..npd+2) does not fit the fluid rows");
  if (!(h.dt > 0.f) || !(h.fpeak > 0.f)) return fail(MFDM_ERR_ARG, "dt and fpeak must be > 0");
  if (h.nt < 0) return fail(MFDM_ERR_ARG, "nt must be >= 0");
  if (h.snapshot <= 0) return fail(MFDM_ERR_ARG, "snapshot interval must be > 0");
  if (h.srcx.size() != h.srcz.size()) return fail(MFDM_ERR_ARG, "posx/posz length mismatch");
  const HostModel::View& v = h.v;
  if (!v.K || !v.rhof || !v.C11 || !v.C13 || !v.C33 || !v.C55 || !v.rhos || !v.J || !v.xix ||
      !v.xiz || !v.zex || !v.zez)
    return fail(MFDM_ERR_ARG, "null model array");
  return MFDM_OK;
}

// CFS-PML profile of one axis in FP64: every cell through mfdm::pml_cell.
void pml_profile(const HostModel& h, int n, bool lo, bool hi, float fpeak, float beta0,
                 std::vector<float4>& out) {
  out.resize(size_t(n));
  for (int i = 0; i < n; ++i)
    out[size_t(i)] = mfdm::pml_cell(fpeak, beta0, h.npd, h.npow, h.vp_max, h.rc, h.thickness, i, n,
                                    lo, hi);
}

int read_bin(const std::string& path, size_t count, std::vector<float>& out) {
  out.resize(count);
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return fail(MFDM_ERR_IO, "Failed to open file: " + path);
  const size_t got = std::fread(out.data(), sizeof(float), count, f);
  std::fclose(f);
  if (got != count) return fail(MFDM_ERR_IO, "Failed to read data from file: " + path);
  return MFDM_OK;
}

// Reads the JSON schema of json_template.json (src/elements.cu:64-176).
int load_json(const char* path, HostModel& h) {
  try {
    const mfdm::JsonConfig J = mfdm::JsonConfig::from_file(path);
    h.fpeak = J.get_float("base.fpeak");
    h.dt = J.get_float("base.dt");
    h.nt = J.get_int("base.nt");
    h.snapshot = J.get_int("base.snapshot");
    const int calc_type = J.get_int("grid.calc_type");
    const int bdy = J.get_int("grid.boundary_type");
    if (calc_type != 1 || (bdy != 1 && bdy != 2))
      return fail(MFDM_ERR_ARG,
                  "unsupported configuration: only calc_type 1 (fluid over solid) with "
                  "boundary_type 2 (CFS-PML sides and bottom, free surface on top) or 1 "
                  "(CFS-PML on all four sides)");
    h.bdy = bdy;
    const size_t nsrc = J.size("grid.src_pos.posx");
    for (size_t i = 0; i < nsrc; ++i) {
      h.srcx.push_back(J.get_int("grid.src_pos.posx", i));
      h.srcz.push_back(J.get_int("grid.src_pos.posz", i));
    }
    h.nx = J.get_int("grid.solid.nx");
    h.nzs = J.get_int("grid.solid.nz");
    const int nxf = J.get_int("grid.fluid.nx");
    h.nzf = J.get_int("grid.fluid.nz");
    if (nxf != h.nx) return fail(MFDM_ERR_CONFIG, "nx_fluid doesn't match nx_solid!");
    h.npd = J.get_int("PML.npd");
    h.thickness = J.get_float("PML.thickness");
    h.npow = J.get_int("PML.NPOW");
    h.vp_max = J.get_float("PML.Vp_max");
    h.rc = J.get_float("PML.Rc");
    h.beta0 = J.get_float("PML.beta0");
    if (h.nx <= 0 || h.nzf <= 0 || h.nzs <= 0) return fail(MFDM_ERR_CONFIG, "bad grid size");
    const size_t nf = size_t(h.nx) * h.nzf, ns = size_t(h.nx) * h.nzs,
                 ng = size_t(h.nx) * (h.nzf + h.nzs - 1);
    struct Item { const char* key; std::vector<float>* dst; size_t n; } items[] = {
        {"grid.solid.C11", &h.C11, ns}, {"grid.solid.C13", &h.C13, ns},
        {"grid.solid.C33", &h.C33, ns}, {"grid.solid.C55", &h.C55, ns},
        {"grid.solid.rho", &h.rhos, ns}, {"grid.fluid.K", &h.K, nf},
        {"grid.fluid.rho", &h.rhof, nf}, {"grid.jacob.J", &h.J, ng},
        {"grid.jacob.xi_x", &h.xix, ng}, {"grid.jacob.xi_z", &h.xiz, ng},
        {"grid.jacob.ze_x", &h.zex, ng}, {"grid.jacob.ze_z", &h.zez, ng}};
    for (const Item& it : items) {
      const int rc = read_bin(J.get_string(it.key), it.n, *it.dst);
      if (rc != MFDM_OK) return rc;
    }
    h.view_own();
  } catch (const std::exception& e) {
    return fail(MFDM_ERR_CONFIG, e.what());
  }
  return MFDM_OK;
}

void fill_src_table(const HostModel& h, float fpeak, int steps, float* amp) {
  const float dt = h.dt;
  const float half = float(double(dt) * 0.5);
  for (int it = 0; it < steps; ++it) {
    const float t = float(it) * dt;  // `const float time = it * mem.dt` (src/pml_fs_kernels.cu:770)
    amp[size_t(it) * 4 + 0] = ricker_ref(fpeak, t);
    amp[size_t(it) * 4 + 1] = ricker_ref(fpeak, t + half);
    amp[size_t(it) * 4 + 2] = ricker_ref(fpeak, t + half);
    amp[size_t(it) * 4 + 3] = ricker_ref(fpeak, t + dt);
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// Map of a block [nf][rows][P] of floats read in boxes of box_x columns, kStageR
// rows and all nf fields. Point-wise maps land as [field][row][col] (dimensions
// column, row, field); stencil maps (rows_outer) land as [row][field][col]
// (dimensions column, field, row), so consecutive chunks stack into one
// row-contiguous ring.
// With nshots > 0 the map has a fourth dimension, the shot, of stride shot_bytes.
int encode_block(CUtensorMap* map, const float* base, int P, int rows, int nf, int box_x,
                 bool rows_outer, int nshots = 0, size_t shot_bytes = 0) {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    MFDM_CU(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess)
      return fail(MFDM_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  const cuuint64_t row_stride = cuuint64_t(P) * 4, field_stride = cuuint64_t(rows) * P * 4;
  const cuuint64_t dims[4] = {cuuint64_t(P), cuuint64_t(rows_outer ? nf : rows),
                              cuuint64_t(rows_outer ? rows : nf), cuuint64_t(nshots > 0 ? nshots : 1)};
  const cuuint64_t strides[3] = {rows_outer ? field_stride : row_stride,
                                 rows_outer ? row_stride : field_stride, cuuint64_t(shot_bytes)};
  const cuuint32_t box[4] = {cuuint32_t(box_x), cuuint32_t(rows_outer ? nf : mfdm::kStageR),
                             cuuint32_t(rows_outer ? mfdm::kStageR : nf), 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, nshots > 0 ? 4 : 3,
                        const_cast<float*>(base), dims,
                        strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(MFDM_ERR_CUDA, "tensor map encoding failed (" + std::to_string(int(r)) + ")");
  return MFDM_OK;
}

void release_graph(mfdm_model* m) {
  ++m->gen;
  if (m->graph) {
    cudaGraphExecDestroy(m->graph);
    m->graph = nullptr;
  }
}

// Grows the source table and the receiver buffer so that steps up to `steps` fit.
int ensure_capacity(mfdm_model* m, int steps) {
  if (steps > m->src_steps) {
    const int cap = std::max(steps, m->src_steps * 2);
    std::vector<float> amp(size_t(m->nshots) * cap * 4, 0.f);  // [shot][step][stage]
    for (int b = 0; b < m->nshots; ++b)
      fill_src_table(m->cfg, m->shots[size_t(b)].fpeak, cap, amp.data() + size_t(b) * cap * 4);
    float* d = nullptr;
    MFDM_CU(cudaMalloc(&d, amp.size() * sizeof(float)));
    MFDM_CU(cudaMemcpy(d, amp.data(), amp.size() * sizeof(float), cudaMemcpyHostToDevice));
    if (m->d_src) cudaFree(m->d_src);
    m->d_src = d;
    m->src_steps = cap;
    m->C.src_stride = size_t(cap) * 4;
    release_graph(m);
  }
  const int need = (steps + m->gap - 1) / m->gap;
  if (need > m->rec_cap) {
    const int cap = std::max(need, m->rec_cap * 2);
    const size_t row = size_t(3) * m->cfg.nx * sizeof(float);  // [shot][sample][3][nx]
    float* d = nullptr;
    MFDM_CU(cudaMalloc(&d, size_t(m->nshots) * cap * row));
    MFDM_CU(cudaMemsetAsync(d, 0, size_t(m->nshots) * cap * row, m->stream));
    if (m->d_rec) {
      MFDM_CU(cudaMemcpy2DAsync(d, size_t(cap) * row, m->d_rec, size_t(m->rec_cap) * row,
                                size_t(m->rec_cap) * row, size_t(m->nshots),
                                cudaMemcpyDeviceToDevice, m->stream));
      MFDM_CU(cudaStreamSynchronize(m->stream));
      cudaFree(m->d_rec);
    }
    m->d_rec = d;
    m->rec_cap = cap;
    m->C.rec_stride = size_t(cap) * 3 * m->cfg.nx;
    release_graph(m);
  }
  m->C.src_amp = m->d_src;
  m->C.src_steps = m->src_steps;
  m->C.rec = m->d_rec;
  m->C.rec_cap = m->rec_cap;
  return MFDM_OK;
}

// Enqueues the five launches of one step. With `ev` (6 events) an event is
// recorded before the first launch and after every launch.
int enqueue_step(mfdm_model* m, int it, cudaStream_t st, cudaEvent_t* ev = nullptr) {
  const int d0 = (it & 1) ? mfdm::kDirB : mfdm::kDirF, d1 = 1 - d0;
  const Fields &U = m->S[0], &A = m->S[1], &B = m->S[2], &Acc = m->S[3];
  const Coef& C = m->C;
  // stage s reads in[s] and writes out[s]: U -> A -> B -> A -> U
  const Fields* in[4] = {&U, &A, &B, &A};
  const Fields* out[4] = {&A, &B, &A, &U};
  const int in_set[4] = {0, 1, 2, 1};
  const int dir[4] = {d0, d1, d0, d1};
  if (ev) MFDM_CU(cudaEventRecord(ev[0], st));
  for (int s = 0; s < 4; ++s) {
    mfdm::StageMaps maps;
    maps.fin = m->fst[in_set[s]];
    maps.sin = m->sst[in_set[s]];
    maps.fun = m->fpw[0];
    maps.sun = m->spw[0];
    maps.facc = m->fpw[3];
    maps.sacc = m->spw[3];
    maps.fcoef = m->fco;
    maps.scoef = m->sco;
    MFDM_CU(mfdm::launch_stage(C, *in[s], *out[s], U, Acc, maps, s, dir[s], st));
    if (ev) MFDM_CU(cudaEventRecord(ev[s + 1], st));
  }
  MFDM_CU(mfdm::launch_finish(C, U, st));
  if (ev) MFDM_CU(cudaEventRecord(ev[5], st));
  return MFDM_OK;
}

// Enqueues `nsteps` steps from host_step: graph replays where possible.
int enqueue_steps(mfdm_model* m, int nsteps);

int capture_graph(mfdm_model* m) {
  cudaGraph_t g = nullptr;
  MFDM_CU(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
  int rc = MFDM_OK;
  for (int k = 0; k < kGraphSteps && rc == MFDM_OK; ++k) rc = enqueue_step(m, k, m->stream);
  cudaError_t e = cudaStreamEndCapture(m->stream, &g);
  if (rc != MFDM_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(MFDM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&m->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(MFDM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  return MFDM_OK;
}

// Maps a kernel status word to an error: bit 2 (value 2) is a pipeline wait
// that timed out, after which the handle's state is undefined (reopen it);
// bit 1 a non-finite value.
int status_error(int st, const char* nonfinite_msg) {
  if (st & 2)
    return fail(MFDM_ERR_CUDA,
                "a stage kernel pipeline wait timed out; the handle's state is undefined, reopen it");
  if (st) return fail(MFDM_ERR_NONFINITE, nonfinite_msg);
  return MFDM_OK;
}

int check_status(mfdm_model* m) {
  int st = 0;
  MFDM_CU(cudaMemcpy(&st, m->C.status, sizeof(int), cudaMemcpyDeviceToHost));
  return status_error(st, "non-finite values reached the interface rows");
}

// Uploads the model arrays, the FP64-derived PML tables and normals, and the
// scalars of `h` into the buffers of `m` (shape already checked).
int upload_model(mfdm_model* m, const HostModel& h) {
  const int nx = h.nx, nzf = h.nzf, nzs = h.nzs, nz = nzf + nzs - 1, P = m->P;
  const HostModel::View& v = h.v;
  Coef& C = m->C;
  // Host [rows][nx] -> device [rows][P], straight from the caller's memory
  // (full PCIe rate when the caller's buffers are pinned).
  auto up = [&](const float* dst_c, const float* src, int rows) -> int {
    MFDM_CU(cudaMemcpy2DAsync(const_cast<float*>(dst_c), size_t(P) * sizeof(float), src,
                              size_t(nx) * sizeof(float), size_t(nx) * sizeof(float), size_t(rows),
                              cudaMemcpyHostToDevice, m->stream));
    return MFDM_OK;
  };
  int rc;
  if ((rc = up(C.K, v.K, nzf)) || (rc = up(C.rhof, v.rhof, nzf)) || (rc = up(C.C11, v.C11, nzs)) ||
      (rc = up(C.C13, v.C13, nzs)) || (rc = up(C.C33, v.C33, nzs)) ||
      (rc = up(C.C55, v.C55, nzs)) || (rc = up(C.rhos, v.rhos, nzs)) || (rc = up(C.J, v.J, nz)) ||
      (rc = up(C.xix, v.xix, nz)) || (rc = up(C.xiz, v.xiz, nz)) || (rc = up(C.zex, v.zex, nz)) ||
      (rc = up(C.zez, v.zez, nz)))
    return rc;
#if MFDM_RCP_RHO
  // density slots hold 1/rho (reciprocal in FP64, rounded once), formed on the device
  MFDM_CU(mfdm::launch_reciprocal(const_cast<float*>(C.rhof), nzf, nx, P, m->stream));
  MFDM_CU(mfdm::launch_reciprocal(const_cast<float*>(C.rhos), nzs, nx, P, m->stream));
#endif
  // Per-medium copies of the metric for the streamed coefficient blocks: fluid
  // rows are global rows 0..nz_f-1, solid rows are global rows nz_f-1..nz-1
  // (device to device, from the global-row metric just uploaded).
  const size_t nfe = size_t(nzf) * P, nse = size_t(nzs) * P, pitch = size_t(P) * sizeof(float);
  const float* met[4] = {C.xix, C.xiz, C.zex, C.zez};
  for (int q = 0; q < 4; ++q) {
    MFDM_CU(cudaMemcpy2DAsync(m->fcoef + q * nfe, pitch, met[q], pitch, pitch, size_t(nzf),
                              cudaMemcpyDeviceToDevice, m->stream));
    MFDM_CU(cudaMemcpy2DAsync(m->scoef + q * nse, pitch, met[q] + size_t(nzf - 1) * P, pitch, pitch,
                              size_t(nzs), cudaMemcpyDeviceToDevice, m->stream));
  }
  if (!m->batch) {  // a plain handle's single shot follows the model's frequency
    m->shots.resize(1);
    m->shots[0].fpeak = h.fpeak;
    m->shots[0].beta0 = h.beta0;
  }
  // Interface unit normal n = grad(zeta)/|grad(zeta)| in FP64 (src/elements.cu:892-905).
  std::vector<float2> nrm(static_cast<size_t>(nx));
  for (int ix = 0; ix < nx; ++ix) {
    const size_t i = size_t(nzf - 1) * nx + ix;
    const double a = v.zex[i], b = v.zez[i], s = std::sqrt(a * a + b * b);
    nrm[size_t(ix)] = s > 0 ? make_float2(float(a / s), float(b / s)) : make_float2(0.f, 1.f);
  }
  MFDM_CU(cudaMemcpyAsync(const_cast<float2*>(C.nrm), nrm.data(), nrm.size() * sizeof(float2),
                          cudaMemcpyHostToDevice, m->stream));
  // CFS-PML factors per shot (alpha0 and beta0 follow the shot's frequency)
  for (int b = 0; b < m->nshots; ++b) {
    std::vector<float4> px, pz;
    const ShotCfg& sh = m->shots[size_t(b)];
    pml_profile(h, nx, true, true, sh.fpeak, sh.beta0, px);
    pml_profile(h, nzs, false, true, sh.fpeak, sh.beta0, pz);
    std::vector<float4> pzf;  // fluid rows: a top band with four-side CPML (elements.cu:866-869)
    pml_profile(h, nzf, h.bdy == 1, false, sh.fpeak, sh.beta0, pzf);
    const size_t so = size_t(b) * C.shot_stride;
    MFDM_CU(cudaMemcpyAsync(const_cast<float*>(reinterpret_cast<const float*>(C.pmlzf)) + so, pzf.data(),
                            pzf.size() * sizeof(float4), cudaMemcpyHostToDevice, m->stream));
    MFDM_CU(cudaMemcpyAsync(const_cast<float*>(reinterpret_cast<const float*>(C.pmlx)) + so, px.data(),
                            px.size() * sizeof(float4), cudaMemcpyHostToDevice, m->stream));
    MFDM_CU(cudaMemcpyAsync(const_cast<float*>(reinterpret_cast<const float*>(C.pmlz)) + so, pz.data(),
                            pz.size() * sizeof(float4), cudaMemcpyHostToDevice, m->stream));
  }
  MFDM_CU(cudaStreamSynchronize(m->stream));

  const float dt = h.dt;
  // RK4 coefficients exactly as the reference forms them in float (src/pml_fs_kernels.cu:735,781-806).
  C.rk_c[0] = dt / 2; C.rk_c[1] = dt / 2; C.rk_c[2] = dt; C.rk_c[3] = dt / 6.0f;
  C.rk_w[0] = dt / 6; C.rk_w[1] = dt / 3; C.rk_w[2] = dt / 3;
  m->gap = std::max(1, int(1e-3 / double(h.dt) + 0.5));  // src/main.cu:92
  C.gap = m->gap;
  // Keep the scalars only.
  HostModel& c = m->cfg;
  c.nx = h.nx; c.nzf = h.nzf; c.nzs = h.nzs;
  c.fpeak = h.fpeak; c.dt = h.dt; c.nt = h.nt; c.snapshot = h.snapshot;
  c.npd = h.npd; c.npow = h.npow; c.thickness = h.thickness;
  c.vp_max = h.vp_max; c.rc = h.rc; c.beta0 = h.beta0; c.bdy = h.bdy;
  c.srcx = h.srcx; c.srcz = h.srcz;
  if (m->isrc >= int(c.srcx.size())) m->isrc = 0;
  C.srcx = c.srcx.empty() ? -1 : c.srcx[size_t(m->isrc)];
  C.srcz = c.srcx.empty() ? 0 : c.srcz[size_t(m->isrc)];
  // The source table depends on fpeak and dt: rebuild it.
  if (m->d_src) cudaFree(m->d_src);
  m->d_src = nullptr;
  m->src_steps = 0;
  release_graph(m);
  return ensure_capacity(m, std::max(h.nt, 1));
}

// Carves every fixed-size device buffer out of one allocation and uploads the model.
// `shots` (batch handles): the shots stepped together; nullptr for a plain handle.
int build(mfdm_model* m, HostModel&& h, int device, const std::vector<ShotCfg>* shots = nullptr) {
  int rc = validate(h);
  if (rc != MFDM_OK) return rc;
  if (shots) {
    if (shots->empty()) return fail(MFDM_ERR_ARG, "a batch needs at least one shot");
    for (const ShotCfg& sh : *shots) {
      if (!(sh.fpeak > 0.f) || !(sh.beta0 >= 1.f))
        return fail(MFDM_ERR_ARG, "each shot needs fpeak > 0 and beta0 >= 1");
      if (sh.x >= 0 && (sh.x >= h.nx || sh.z < 0 || sh.z >= h.nzf))
        return fail(MFDM_ERR_ARG, "shot source outside the fluid grid");
    }
    m->batch = true;
    m->shots = *shots;
  } else {
    m->batch = false;
    m->shots.assign(1, ShotCfg{});
  }
  m->nshots = int(m->shots.size());
  m->device = device;
  int ndev = 0;
  MFDM_CU(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(MFDM_ERR_ARG, "no such CUDA device");
  MFDM_CU(cudaSetDevice(device));
  MFDM_CU(mfdm::configure_device());
  MFDM_CU(mfdm::upload_constants(kSrcW, kW7));
  MFDM_CU(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));

  const int nx = h.nx, nzf = h.nzf, nzs = h.nzs, nz = nzf + nzs - 1;
  // pitch: 128-byte rows, and never narrower than the 72-column TMA stencil box
  const int P = round_up(std::max(nx, mfdm::kStageSW), 32), Ps = round_up(std::max(2 * h.npd, 1), 4);
  const int npdr = std::max(h.npd, 1);
  m->P = P; m->Ps = Ps; m->nz = nz;

  // Byte offsets of every buffer (256-byte aligned).
  size_t off = 0;
  auto take = [&](size_t nfloats) {
    const size_t o = off;
    off += (nfloats * sizeof(float) + 255) / 256 * 256;
    return o;
  };
  const size_t nf = size_t(nzf) * P, ns = size_t(nzs) * P, ng = size_t(nz) * P;
  const size_t o_fco = take(6 * nf), o_sco = take(9 * ns);
  const size_t o_J = take(ng), o_xix = take(ng), o_xiz = take(ng), o_zex = take(ng),
               o_zez = take(ng);
  const size_t o_nrm = take(size_t(nx) * 2), o_misc = take(64),
               o_srcpos = take(size_t(2) * m->nshots);
  const size_t shared = off;
  // One region per shot (equal sizes, so shot b's buffers are b regions after
  // shot 0's): each RK set's fluid block [3][nz_f][P] and solid block
  // [5][nz_s][P] (the TMA boxes span the fields), the ADE strips, the PML
  // factors and the interface rows.
  size_t roff = 0;
  auto rtake = [&](size_t nfloats) {
    const size_t o = roff;
    roff += (nfloats * sizeof(float) + 255) / 256 * 256;
    return o;
  };
  size_t o_fb[4], o_sb[4], o_ade[4][12], o_fza[4][4];
  for (int s = 0; s < 4; ++s) {
    o_fb[s] = rtake(3 * nf);
    o_sb[s] = rtake(5 * ns);
    for (int q = 0; q < 4; ++q) o_ade[s][q] = rtake(size_t(nzf) * Ps);
    for (int q = 0; q < 4; ++q) o_ade[s][4 + q] = rtake(size_t(nzs) * Ps);
    for (int q = 0; q < 4; ++q) o_ade[s][8 + q] = rtake(size_t(npdr) * P);
    for (int q = 0; q < 4; ++q) o_fza[s][q] = rtake(h.bdy == 1 ? size_t(npdr) * P : 1);
  }
  const size_t o_pmlx = rtake(size_t(nx) * 4), o_pmlz = rtake(size_t(nzs) * 4),
               o_pmlzf = rtake(size_t(nzf) * 4), o_ipre = rtake(size_t(8) * P);
  m->region = roff;
  off = shared + roff * size_t(m->nshots);
  m->dbytes = off;
  MFDM_CU(cudaMalloc(&m->dmem, off));
  MFDM_CU(cudaMemsetAsync(m->dmem, 0, off, m->stream));
  char* base = m->dmem;
  auto F = [&](size_t o) { return reinterpret_cast<float*>(base + o); };
  auto R = [&](size_t o) { return reinterpret_cast<float*>(base + shared + o); };  // shot 0
  for (int s = 0; s < 4; ++s) {
    Fields& S = m->S[s];
    float* fb = R(o_fb[s]);
    float* sb = R(o_sb[s]);
    S.fvx = fb; S.fvz = fb + nf; S.fp = fb + 2 * nf;
    S.svx = sb; S.svz = sb + ns; S.ssx = sb + 2 * ns; S.ssz = sb + 3 * ns; S.ssxz = sb + 4 * ns;
    for (int q = 0; q < 4; ++q) {
      S.fx[q] = R(o_ade[s][q]);
      S.sx[q] = R(o_ade[s][4 + q]);
      S.sz[q] = R(o_ade[s][8 + q]);
      S.fz[q] = R(o_fza[s][q]);
    }
  }
  m->fcoef = F(o_fco);
  m->scoef = F(o_sco);
  Coef& C = m->C;
  C.nx = nx; C.nzf = nzf; C.nzs = nzs; C.P = P; C.npd = h.npd; C.Ps = Ps;
  C.rhof = m->fcoef + 4 * nf; C.K = m->fcoef + 5 * nf;
  C.rhos = m->scoef + 4 * ns; C.C11 = m->scoef + 5 * ns; C.C13 = m->scoef + 6 * ns;
  C.C33 = m->scoef + 7 * ns; C.C55 = m->scoef + 8 * ns;
  C.J = F(o_J); C.xix = F(o_xix); C.xiz = F(o_xiz); C.zex = F(o_zex); C.zez = F(o_zez);
  C.pmlx = reinterpret_cast<const float4*>(R(o_pmlx));
  C.pmlz = reinterpret_cast<const float4*>(R(o_pmlz));
  C.pmlzf = reinterpret_cast<const float4*>(R(o_pmlzf));
  C.cpml = h.bdy == 1 ? 1 : 0;
  C.nrm = reinterpret_cast<const float2*>(F(o_nrm));
  C.ipre = R(o_ipre);
  int* misc = reinterpret_cast<int*>(F(o_misc));
  C.step = misc;
  C.done = reinterpret_cast<unsigned*>(misc + 1);
  C.status = misc + 2;
  C.nshots = m->nshots;
  C.shot_stride = roff / sizeof(float);
  C.src_stride = 0;
  C.rec_stride = 0;
  C.src_pos = nullptr;
  if (m->batch) {
    m->d_srcpos = reinterpret_cast<int*>(F(o_srcpos));
    std::vector<int> pos(size_t(2) * m->nshots);
    for (int b = 0; b < m->nshots; ++b) {
      pos[size_t(2 * b)] = m->shots[size_t(b)].x;
      pos[size_t(2 * b + 1)] = m->shots[size_t(b)].z;
    }
    MFDM_CU(cudaMemcpyAsync(m->d_srcpos, pos.data(), pos.size() * sizeof(int),
                            cudaMemcpyHostToDevice, m->stream));
    C.src_pos = reinterpret_cast<const int2*>(m->d_srcpos);
  }
  for (int s = 0; s < 4; ++s) {
    if ((rc = encode_block(&m->fst[s], R(o_fb[s]), P, nzf, 3, mfdm::kStageSW, true, m->nshots, roff)) ||
        (rc = encode_block(&m->sst[s], R(o_sb[s]), P, nzs, 5, mfdm::kStageSW, true, m->nshots, roff)) ||
        (rc = encode_block(&m->fpw[s], R(o_fb[s]), P, nzf, 3, mfdm::kStageTX, false, m->nshots, roff)) ||
        (rc = encode_block(&m->spw[s], R(o_sb[s]), P, nzs, 5, mfdm::kStageTX, false, m->nshots, roff)))
      return rc;
  }
  if ((rc = encode_block(&m->fco, m->fcoef, P, nzf, 6, mfdm::kStageTX, false)) ||
      (rc = encode_block(&m->sco, m->scoef, P, nzs, 9, mfdm::kStageTX, false)))
    return rc;
  if ((rc = upload_model(m, h)) != MFDM_OK) return rc;
  MFDM_CU(mfdm::launch_set_step(m->C, 0, m->stream));
  MFDM_CU(cudaStreamSynchronize(m->stream));
  return MFDM_OK;
}

void destroy(mfdm_model* m) {
  if (!m) return;
  DeviceGuard g(m->device);
  release_graph(m);
  if (m->stream) cudaStreamSynchronize(m->stream);
  if (m->d_src) cudaFree(m->d_src);
  if (m->d_rec) cudaFree(m->d_rec);
  if (m->dmem) cudaFree(m->dmem);
  delete m->adj;
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

int open_common(HostModel&& h, int device, mfdm_model** out,
                const std::vector<ShotCfg>* shots = nullptr) {
  if (!out) return fail(MFDM_ERR_ARG, "null output handle");
  *out = nullptr;
  int prev = -1;
  cudaGetDevice(&prev);
  mfdm_model* m = new mfdm_model();
  const int rc = build(m, std::move(h), device, shots);
  if (prev >= 0) cudaSetDevice(prev);
  if (rc != MFDM_OK) {
    const std::string msg = g_err;
    destroy(m);
    g_err = msg;
    return rc;
  }
  *out = m;
  return MFDM_OK;
}

int field_ptr(mfdm_model* m, int field, float** p, int* rows, int shot = 0);

// Zeroes every shot's RK sets (state, stage buffers, accumulator), ADE strips
// and interface rows; the coefficients and the PML tables stay.
int clear_state(mfdm_model* m) {
  const size_t pitch = m->region, h = size_t(m->nshots);
  const size_t nf = size_t(m->cfg.nzf) * m->P, ns = size_t(m->cfg.nzs) * m->P;
  for (int s = 0; s < 4; ++s) {
    const Fields& S = m->S[s];
    MFDM_CU(cudaMemset2DAsync(S.fvx, pitch, 0, 3 * nf * sizeof(float), h, m->stream));
    MFDM_CU(cudaMemset2DAsync(S.svx, pitch, 0, 5 * ns * sizeof(float), h, m->stream));
    for (int q = 0; q < 4; ++q) {
      MFDM_CU(cudaMemset2DAsync(S.fx[q], pitch, 0, size_t(m->cfg.nzf) * m->Ps * sizeof(float), h,
                                m->stream));
      MFDM_CU(cudaMemset2DAsync(S.sx[q], pitch, 0, size_t(m->cfg.nzs) * m->Ps * sizeof(float), h,
                                m->stream));
      MFDM_CU(cudaMemset2DAsync(S.sz[q], pitch, 0,
                                size_t(std::max(m->cfg.npd, 1)) * m->P * sizeof(float), h, m->stream));
      if (m->C.cpml)
        MFDM_CU(cudaMemset2DAsync(S.fz[q], pitch, 0,
                                  size_t(std::max(m->cfg.npd, 1)) * m->P * sizeof(float), h,
                                  m->stream));
    }
  }
  MFDM_CU(cudaMemset2DAsync(m->C.ipre, pitch, 0, size_t(8) * m->P * sizeof(float), h, m->stream));
  return MFDM_OK;
}

// Clears the receiver rows and the error word and rewinds the step counter.
int rewind(mfdm_model* m) {
  MFDM_CU(cudaMemsetAsync(m->d_rec, 0,
                          size_t(m->nshots) * m->rec_cap * 3 * m->cfg.nx * sizeof(float), m->stream));
  MFDM_CU(cudaMemsetAsync(m->C.status, 0, sizeof(int), m->stream));
  m->host_step = 0;
  MFDM_CU(mfdm::launch_set_step(m->C, 0, m->stream));
  MFDM_CU(cudaStreamSynchronize(m->stream));
  return MFDM_OK;
}

int get_records(mfdm_model* m, int shot, int first, int count, float* svx, float* svz, float* fp) {
  if (shot < 0 || shot >= m->nshots) return fail(MFDM_ERR_ARG, "shot index out of range");
  const int avail = (m->host_step + m->gap - 1) / m->gap;
  if (first < 0 || count < 0 || first + count > avail || first + count > m->rec_cap)
    return fail(MFDM_ERR_ARG, "record range out of bounds");
  if (count == 0) return MFDM_OK;
  DeviceGuard g(m->device);
  const int nx = m->cfg.nx;
  const float* rec = m->d_rec + size_t(shot) * m->C.rec_stride;
  float* outs[3] = {svx, svz, fp};
  for (int q = 0; q < 3; ++q) {
    if (!outs[q]) continue;
    MFDM_CU(cudaMemcpy2DAsync(outs[q], size_t(nx) * sizeof(float),
                              rec + (size_t(first) * 3 + q) * nx, size_t(3) * nx * sizeof(float),
                              size_t(nx) * sizeof(float), size_t(count), cudaMemcpyDeviceToHost,
                              m->stream));
  }
  MFDM_CU(cudaStreamSynchronize(m->stream));
  return MFDM_OK;
}

int get_field(mfdm_model* m, int shot, int field, float* host) {
  if (!host) return fail(MFDM_ERR_ARG, "null argument");
  float* p = nullptr;
  int rows = 0;
  int rc = field_ptr(m, field, &p, &rows, shot);
  if (rc != MFDM_OK) return rc;
  DeviceGuard g(m->device);
  MFDM_CU(cudaMemcpy2DAsync(host, size_t(m->cfg.nx) * sizeof(float), p, size_t(m->P) * sizeof(float),
                            size_t(m->cfg.nx) * sizeof(float), size_t(rows), cudaMemcpyDeviceToHost,
                            m->stream));
  MFDM_CU(cudaStreamSynchronize(m->stream));
  return MFDM_OK;
}

int field_ptr(mfdm_model* m, int field, float** p, int* rows, int shot) {
  const Fields& U = m->S[0];
  float* const ptrs[8] = {U.fvx, U.fvz, U.fp, U.svx, U.svz, U.ssx, U.ssz, U.ssxz};
  if (field < 0 || field > 7) return fail(MFDM_ERR_ARG, "bad field id");
  if (shot < 0 || shot >= m->nshots) return fail(MFDM_ERR_ARG, "shot index out of range");
  *p = ptrs[field] + size_t(shot) * m->C.shot_stride;
  *rows = field < 3 ? m->cfg.nzf : m->cfg.nzs;
  return MFDM_OK;
}

}  // namespace

namespace mfdm {
// Shared with other translation units of the library.
int set_error(int code, const char* msg) { return fail(code, msg); }
int encode_block_map(CUtensorMap* map, const float* base, int P, int rows, int nf, int box_x,
                     bool rows_outer, int nshots, size_t shot_bytes) {
  return encode_block(map, base, P, rows, nf, box_x, rows_outer, nshots, shot_bytes);
}
}  // namespace mfdm

extern "C" {

const char* mfdm_last_error(void) { return g_err.c_str(); }

int mfdm_open_json(const char* json_path, int device, mfdm_model** out) {
  if (!json_path) return fail(MFDM_ERR_ARG, "null JSON path");
  HostModel h;
  const int rc = load_json(json_path, h);
  if (rc != MFDM_OK) return rc;
  return open_common(std::move(h), device, out);
}

}  // extern "C"

namespace {
int desc_to_host(const mfdm_desc* d, HostModel& h) {
  if (!d) return fail(MFDM_ERR_ARG, "null descriptor");
  h.nx = d->nx; h.nzf = d->nz_f; h.nzs = d->nz_s;
  h.fpeak = d->fpeak; h.dt = d->dt; h.nt = d->nt; h.snapshot = d->snapshot;
  h.npd = d->npd; h.npow = d->npow; h.thickness = d->thickness; h.vp_max = d->vp_max;
  h.rc = d->rc; h.beta0 = d->beta0;
  h.bdy = d->boundary_type == 1 ? 1 : 2;
  if (h.nx <= 0 || h.nzf <= 0 || h.nzs <= 0) return fail(MFDM_ERR_ARG, "bad grid size");
  for (int i = 0; i < d->nsrc; ++i) {
    if (!d->src_x || !d->src_z) return fail(MFDM_ERR_ARG, "null source arrays");
    h.srcx.push_back(d->src_x[i]);
    h.srcz.push_back(d->src_z[i]);
  }
  // the caller's arrays are read in place by the upload (no host copy)
  h.v = {d->K, d->rho_f, d->C11, d->C13, d->C33, d->C55, d->rho_s,
         d->J, d->xi_x, d->xi_z, d->ze_x, d->ze_z};
  return MFDM_OK;
}

int enqueue_steps(mfdm_model* m, int nsteps) {
  int rc;
  while (nsteps > 0) {
    if ((m->host_step & 1) == 0 && nsteps >= kGraphSteps) {
      if (!m->graph && (rc = capture_graph(m)) != MFDM_OK) return rc;
      MFDM_CU(cudaGraphLaunch(m->graph, m->stream));
      m->host_step += kGraphSteps;
      nsteps -= kGraphSteps;
    } else {
      if ((rc = enqueue_step(m, m->host_step, m->stream)) != MFDM_OK) return rc;
      ++m->host_step;
      --nsteps;
    }
  }
  return MFDM_OK;
}
}  // namespace

extern "C" {

int mfdm_open_desc(const mfdm_desc* d, int device, mfdm_model** out) {
  HostModel h;
  const int rc = desc_to_host(d, h);
  if (rc != MFDM_OK) return rc;
  return open_common(std::move(h), device, out);
}

int mfdm_load_desc(mfdm_model* m, const mfdm_desc* d) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  HostModel h;
  int rc = desc_to_host(d, h);
  if (rc != MFDM_OK) return rc;
  if ((rc = validate(h)) != MFDM_OK) return rc;
  if (h.nx != m->cfg.nx || h.nzf != m->cfg.nzf || h.nzs != m->cfg.nzs || h.npd != m->cfg.npd ||
      h.bdy != m->cfg.bdy)
    return fail(MFDM_ERR_ARG, "model shape or boundary type differs from the open handle");
  DeviceGuard g(m->device);
  MFDM_CU(cudaStreamSynchronize(m->stream));
  if (m->adj) {  // the transposed operators hold the old coefficients
    m->adj->built = false;
    m->adj->nsteps = -1;
  }
  return upload_model(m, h);
}

int mfdm_close(mfdm_model* m) {
  destroy(m);
  return MFDM_OK;
}

int mfdm_get_info(const mfdm_model* m, mfdm_info* info) {
  if (!m || !info) return fail(MFDM_ERR_ARG, "null argument");
  info->nx = m->cfg.nx; info->nz_f = m->cfg.nzf; info->nz_s = m->cfg.nzs; info->pitch = m->P;
  info->nt = m->cfg.nt; info->snapshot = m->cfg.snapshot; info->gap = m->gap;
  info->nsrc = int(m->cfg.srcx.size()); info->shot = m->isrc; info->step = m->host_step;
  info->nsamples = (m->host_step + m->gap - 1) / m->gap;
  info->cells = (long long)m->cfg.nx * (m->cfg.nzf + m->cfg.nzs);
  info->device_bytes = (long long)m->dbytes + (long long)m->nshots * m->src_steps * 16 +
                       (long long)m->nshots * m->rec_cap * 12 * m->cfg.nx;
  info->nshots = m->nshots;
  info->seg_rows = mfdm::stage_seg_rows(m->C);
  info->blocks_per_sm = mfdm::stage_blocks_per_sm(m->C);
  return MFDM_OK;
}

int mfdm_set_shot(mfdm_model* m, int isrc, int reset_state) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  if (m->batch) return fail(MFDM_ERR_ARG, "a batch handle runs its own shots: use mfdm_batch_reset");
  if (isrc < 0 || (isrc >= int(m->cfg.srcx.size()) && !m->cfg.srcx.empty()))
    return fail(MFDM_ERR_ARG, "shot index out of range");
  DeviceGuard g(m->device);
  m->isrc = isrc;
  m->C.srcx = m->cfg.srcx.empty() ? -1 : m->cfg.srcx[size_t(isrc)];
  m->C.srcz = m->cfg.srcx.empty() ? 0 : m->cfg.srcz[size_t(isrc)];
  release_graph(m);  // the source position is baked into the kernel arguments
  int rc;
  // every state set, the stage buffers and the accumulator (the coefficient block is untouched)
  if (reset_state && (rc = clear_state(m)) != MFDM_OK) return rc;
  return rewind(m);
}

int mfdm_update_rk4(mfdm_model* m, int it, void* stream) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  if (it < 0) return fail(MFDM_ERR_ARG, "negative time index");
  DeviceGuard g(m->device);
  int rc = ensure_capacity(m, it + 1);
  if (rc != MFDM_OK) return rc;
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : m->stream;
  if (st != m->stream) MFDM_CU(cudaStreamSynchronize(m->stream));
  MFDM_CU(mfdm::launch_set_step(m->C, it, st));
  rc = enqueue_step(m, it, st);
  if (rc != MFDM_OK) return rc;
  m->host_step = it + 1;
  return MFDM_OK;
}

int mfdm_step(mfdm_model* m, int nsteps) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  if (nsteps < 0) return fail(MFDM_ERR_ARG, "negative step count");
  DeviceGuard g(m->device);
  int rc = ensure_capacity(m, m->host_step + nsteps);
  if (rc != MFDM_OK) return rc;
  if ((rc = enqueue_steps(m, nsteps)) != MFDM_OK) return rc;
  MFDM_CU(cudaStreamSynchronize(m->stream));
  return check_status(m);
}

int mfdm_time_steps(mfdm_model* m, int nsteps, int per_kernel, float* total_ms, float* kernel_ms) {
  if (!m || !total_ms || (per_kernel && !kernel_ms)) return fail(MFDM_ERR_ARG, "null argument");
  if (nsteps < 0) return fail(MFDM_ERR_ARG, "negative step count");
  DeviceGuard g(m->device);
  int rc = ensure_capacity(m, m->host_step + nsteps);
  if (rc != MFDM_OK) return rc;
  cudaEvent_t ev[8] = {};
  for (auto& e : ev) MFDM_CU(cudaEventCreate(&e));
  struct Free { cudaEvent_t* e; ~Free() { for (int i = 0; i < 8; ++i) cudaEventDestroy(e[i]); } } fr{ev};
  if (!per_kernel) {
    // the time loop's graph is captured and uploaded before the timed region:
    // a one-time setup (the first mfdm_step of 32 steps or more does it too)
    if (!m->graph && nsteps >= kGraphSteps) {
      if ((rc = capture_graph(m)) != MFDM_OK) return rc;
      if (cudaGraphUpload(m->graph, m->stream) != cudaSuccess) (void)cudaGetLastError();
    }
    MFDM_CU(cudaEventRecord(ev[6], m->stream));
    if ((rc = enqueue_steps(m, nsteps)) != MFDM_OK) return rc;
    MFDM_CU(cudaEventRecord(ev[7], m->stream));
    MFDM_CU(cudaEventSynchronize(ev[7]));
    MFDM_CU(cudaEventElapsedTime(total_ms, ev[6], ev[7]));
    return check_status(m);
  }
  // the steps go back to back (no wait between them, as in a run), in chunks
  // of kChunk steps with six events each
  constexpr int kChunk = 256;
  std::vector<cudaEvent_t> pool(size_t(std::min(nsteps, kChunk)) * 6, nullptr);
  struct FreePool {
    std::vector<cudaEvent_t>& p;
    ~FreePool() { for (cudaEvent_t e : p) if (e) cudaEventDestroy(e); }
  } fp{pool};
  for (auto& e : pool) MFDM_CU(cudaEventCreate(&e));
  float acc[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, tot = 0.f;
  for (int k0 = 0; k0 < nsteps; k0 += kChunk) {
    const int n = std::min(kChunk, nsteps - k0);
    for (int k = 0; k < n; ++k) {
      if ((rc = enqueue_step(m, m->host_step, m->stream, &pool[size_t(k) * 6])) != MFDM_OK) return rc;
      ++m->host_step;
    }
    MFDM_CU(cudaEventSynchronize(pool[size_t(n - 1) * 6 + 5]));
    for (int k = 0; k < n; ++k) {
      const cudaEvent_t* e = &pool[size_t(k) * 6];
      for (int i = 0; i < 5; ++i) {
        float t = 0.f;
        MFDM_CU(cudaEventElapsedTime(&t, e[i], e[i + 1]));
        acc[i] += t;
      }
      float t = 0.f;
      MFDM_CU(cudaEventElapsedTime(&t, e[0], e[5]));
      tot += t;
    }
  }
  for (int i = 0; i < 5; ++i) kernel_ms[i] = acc[i];
  *total_ms = tot;
  return check_status(m);
}

int mfdm_synchronize(mfdm_model* m) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  DeviceGuard g(m->device);
  MFDM_CU(cudaStreamSynchronize(m->stream));
  return check_status(m);
}

int mfdm_get_records(mfdm_model* m, int first, int count, float* svx, float* svz, float* fp) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  return get_records(m, 0, first, count, svx, svz, fp);
}

int mfdm_get_field(mfdm_model* m, int field, float* host) {
  if (!m) return fail(MFDM_ERR_ARG, "null argument");
  return get_field(m, 0, field, host);
}

int mfdm_open_batch(const mfdm_desc* d, int nshots, const mfdm_shot* shots, int device,
                    mfdm_model** out) {
  if (nshots <= 0 || !shots) return fail(MFDM_ERR_ARG, "a batch needs at least one shot");
  HostModel h;
  const int rc = desc_to_host(d, h);
  if (rc != MFDM_OK) return rc;
  std::vector<ShotCfg> sv(static_cast<size_t>(nshots));
  for (int b = 0; b < nshots; ++b) {
    sv[size_t(b)].x = shots[b].src_x;
    sv[size_t(b)].z = shots[b].src_z;
    sv[size_t(b)].fpeak = shots[b].fpeak;
    sv[size_t(b)].beta0 = shots[b].beta0;
  }
  return open_common(std::move(h), device, out, &sv);
}

int mfdm_batch_reset(mfdm_model* m) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  DeviceGuard g(m->device);
  int rc;
  if ((rc = clear_state(m)) != MFDM_OK) return rc;
  return rewind(m);
}

int mfdm_batch_get_records(mfdm_model* m, int shot, int first, int count, float* svx, float* svz,
                           float* fp) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  return get_records(m, shot, first, count, svx, svz, fp);
}

int mfdm_batch_get_field(mfdm_model* m, int shot, int field, float* host) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  return get_field(m, shot, field, host);
}

int mfdm_set_tile(mfdm_model* m, int seg_rows) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  if (seg_rows != 0 && (seg_rows < 4 || seg_rows > 128 || seg_rows % 4 != 0))
    return fail(MFDM_ERR_ARG, "segment rows must be a multiple of 4 in [4, 128] (0: default)");
  DeviceGuard g(m->device);
  MFDM_CU(cudaStreamSynchronize(m->stream));
  m->C.seg = seg_rows;
  release_graph(m);  // the segment height is baked into the captured launches
  return MFDM_OK;
}

}  // extern "C"

namespace {

const int kSegCandidates[] = {8, 12, 16, 24, 32, 48};

std::mutex g_tune_mu;
// (device, nx, nz_f, nz_s, npd, bdy, nshots) -> (rows, blocks per SM)
std::map<std::vector<int>, std::pair<int, int>> g_tune;

// Device time of one captured kGraphSteps-step replay with `seg` rows per segment
// and the stage build of `variant` blocks per SM (after one untimed replay that
// also captures the graph).
int time_segment_rows(mfdm_model* m, int seg, int variant, float* ms) {
  m->C.seg = seg;
  m->C.variant = variant;
  release_graph(m);
  int rc;
  if ((rc = enqueue_steps(m, kGraphSteps)) != MFDM_OK) return rc;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  MFDM_CU(cudaEventCreate(&e0));
  struct Free { cudaEvent_t *a, *b; ~Free() { cudaEventDestroy(*a); if (*b) cudaEventDestroy(*b); } } fr{&e0, &e1};
  MFDM_CU(cudaEventCreate(&e1));
  MFDM_CU(cudaEventRecord(e0, m->stream));
  if ((rc = enqueue_steps(m, kGraphSteps)) != MFDM_OK) return rc;
  MFDM_CU(cudaEventRecord(e1, m->stream));
  MFDM_CU(cudaEventSynchronize(e1));
  MFDM_CU(cudaEventElapsedTime(ms, e0, e1));
  return check_status(m);
}

}  // namespace

extern "C" {

int mfdm_autotune(mfdm_model* m, int* seg_rows) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  DeviceGuard g(m->device);
  const HostModel& h = m->cfg;
  const std::vector<int> key = {m->device, h.nx, h.nzf, h.nzs, h.npd, h.bdy, m->nshots};
  std::pair<int, int> best(0, 0);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) best = it->second;
  }
  int rc;
  if (best.first == 0) {
    // from rest at step 0, so no state of the caller's is stepped
    if ((rc = clear_state(m)) != MFDM_OK) return rc;
    if ((rc = rewind(m)) != MFDM_OK) return rc;
    const int n = int(sizeof(kSegCandidates) / sizeof(int));
    if ((rc = ensure_capacity(m, 2 * kGraphSteps * n * 2)) != MFDM_OK) return rc;
    float best_ms = 0.f;
    for (int variant = 2; variant <= 4; ++variant)
      for (int i = 0; i < n; ++i) {
        if (variant == 4 && kSegCandidates[i] % 8 != 0) continue;  // tile heights: multiples of 8
        float ms = 0.f;
        if ((rc = time_segment_rows(m, kSegCandidates[i], variant, &ms)) != MFDM_OK) return rc;
        if (best.first == 0 || ms < best_ms) {
          best = {kSegCandidates[i], variant};
          best_ms = ms;
        }
      }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = best;
  }
  m->C.seg = best.first;
  m->C.variant = best.second;
  release_graph(m);
  if ((rc = clear_state(m)) != MFDM_OK) return rc;
  if ((rc = rewind(m)) != MFDM_OK) return rc;
  if (seg_rows) *seg_rows = best.first;
  return MFDM_OK;
}

int mfdm_set_blocks_per_sm(mfdm_model* m, int blocks) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  if (blocks != 0 && blocks != 2 && blocks != 3 && blocks != 4)
    return fail(MFDM_ERR_ARG, "stage build must be 2, 3 (blocks per SM), 4 (tiles) or 0 (the default)");
  DeviceGuard g(m->device);
  MFDM_CU(cudaStreamSynchronize(m->stream));
  m->C.variant = blocks;
  release_graph(m);
  return MFDM_OK;
}

}  // extern "C"

// ---- groups of models ---------------------------------------------------------

struct mfdm_group {
  int device = 0;
  std::vector<mfdm_model*> ms;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t graph = nullptr;
  std::vector<unsigned> gens;  // model generations the graph was captured from
};

namespace {

void group_destroy(mfdm_group* g) {
  if (!g) return;
  DeviceGuard d(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  if (g->graph) cudaGraphExecDestroy(g->graph);
  for (cudaEvent_t e : g->join)
    if (e) cudaEventDestroy(e);
  if (g->fork) cudaEventDestroy(g->fork);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

// Enqueues `k` steps of every model on the model's own stream, forked from and
// joined back into the group stream (the models run concurrently). `graph`:
// graph-step indices 0..k-1 (captured), else the models' own time indices.
int group_enqueue(mfdm_group* g, int k, bool graph) {
  MFDM_CU(cudaEventRecord(g->fork, g->stream));
  for (size_t i = 0; i < g->ms.size(); ++i) {
    mfdm_model* m = g->ms[i];
    MFDM_CU(cudaStreamWaitEvent(m->stream, g->fork, 0));
    for (int j = 0; j < k; ++j) {
      const int rc = enqueue_step(m, graph ? j : m->host_step + j, m->stream);
      if (rc != MFDM_OK) return rc;
    }
    MFDM_CU(cudaEventRecord(g->join[i], m->stream));
    MFDM_CU(cudaStreamWaitEvent(g->stream, g->join[i], 0));
  }
  return MFDM_OK;
}

int group_capture(mfdm_group* g) {
  if (g->graph) {
    cudaGraphExecDestroy(g->graph);
    g->graph = nullptr;
  }
  cudaGraph_t gr = nullptr;
  MFDM_CU(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = group_enqueue(g, kGraphSteps, true);
  cudaError_t e = cudaStreamEndCapture(g->stream, &gr);
  if (rc != MFDM_OK) {
    if (gr) cudaGraphDestroy(gr);
    return rc;
  }
  if (e != cudaSuccess) return fail(MFDM_ERR_CUDA, std::string("group capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&g->graph, gr, 0);
  cudaGraphDestroy(gr);
  if (e != cudaSuccess)
    return fail(MFDM_ERR_CUDA, std::string("group instantiate: ") + cudaGetErrorString(e));
  g->gens.clear();
  for (mfdm_model* m : g->ms) g->gens.push_back(m->gen);
  return MFDM_OK;
}

int group_run(mfdm_group* g, int nsteps) {
  if (nsteps < 0) return fail(MFDM_ERR_ARG, "negative step count");
  const int t0 = g->ms[0]->host_step;
  int rc;
  for (mfdm_model* m : g->ms)
    if (m->host_step != t0) return fail(MFDM_ERR_ARG, "grouped models are at different time indices");
  // buffer growth enqueues on the model streams; a graph launched on the
  // group stream would not wait for it
  for (mfdm_model* m : g->ms) {
    if ((rc = ensure_capacity(m, t0 + nsteps)) != MFDM_OK) return rc;
    MFDM_CU(cudaStreamSynchronize(m->stream));
  }
  while (nsteps > 0) {
    const int step = g->ms[0]->host_step;
    int k = 1;
    if ((step & 1) == 0 && nsteps >= kGraphSteps) {
      bool stale = !g->graph;
      for (size_t i = 0; i < g->ms.size() && !stale; ++i) stale = g->gens[i] != g->ms[i]->gen;
      if (stale && (rc = group_capture(g)) != MFDM_OK) return rc;
      MFDM_CU(cudaGraphLaunch(g->graph, g->stream));
      k = kGraphSteps;
    } else if ((rc = group_enqueue(g, 1, false)) != MFDM_OK) {
      return rc;
    }
    for (mfdm_model* m : g->ms) m->host_step += k;
    nsteps -= k;
  }
  return MFDM_OK;
}

int group_check(mfdm_group* g) {
  MFDM_CU(cudaStreamSynchronize(g->stream));
  for (mfdm_model* m : g->ms) {
    const int rc = check_status(m);
    if (rc != MFDM_OK) return rc;
  }
  return MFDM_OK;
}

}  // namespace

extern "C" {

int mfdm_group_open(mfdm_model* const* models, int n, mfdm_group** out) {
  if (!out) return fail(MFDM_ERR_ARG, "null output handle");
  *out = nullptr;
  if (!models || n <= 0) return fail(MFDM_ERR_ARG, "a group needs at least one model");
  mfdm_group* g = new mfdm_group();
  g->device = models[0] ? models[0]->device : 0;
  for (int i = 0; i < n; ++i) {
    if (!models[i]) {
      delete g;
      return fail(MFDM_ERR_ARG, "null model handle in group");
    }
    if (models[i]->device != g->device) {
      delete g;
      return fail(MFDM_ERR_ARG, "grouped models must be on one device");
    }
    for (int j = 0; j < i; ++j)
      if (models[j] == models[i]) {
        delete g;
        return fail(MFDM_ERR_ARG, "a model appears twice in the group");
      }
    g->ms.push_back(models[i]);
  }
  DeviceGuard d(g->device);
  auto cu = [&](cudaError_t e) {
    if (e == cudaSuccess) return true;
    fail(MFDM_ERR_CUDA, std::string("group setup: ") + cudaGetErrorString(e));
    return false;
  };
  bool ok = cu(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking)) &&
            cu(cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming));
  g->join.assign(size_t(n), nullptr);
  for (int i = 0; ok && i < n; ++i) ok = cu(cudaEventCreateWithFlags(&g->join[size_t(i)], cudaEventDisableTiming));
  if (!ok) {
    const std::string msg = g_err;
    group_destroy(g);
    g_err = msg;
    return MFDM_ERR_CUDA;
  }
  *out = g;
  return MFDM_OK;
}

int mfdm_group_step(mfdm_group* g, int nsteps) {
  if (!g) return fail(MFDM_ERR_ARG, "null group");
  DeviceGuard d(g->device);
  const int rc = group_run(g, nsteps);
  if (rc != MFDM_OK) return rc;
  return group_check(g);
}

int mfdm_group_time_steps(mfdm_group* g, int nsteps, float* total_ms) {
  if (!g || !total_ms) return fail(MFDM_ERR_ARG, "null argument");
  DeviceGuard d(g->device);
  cudaEvent_t e[2] = {};
  MFDM_CU(cudaEventCreate(&e[0]));
  struct Free { cudaEvent_t* e; ~Free() { for (int i = 0; i < 2; ++i) if (e[i]) cudaEventDestroy(e[i]); } } fr{e};
  MFDM_CU(cudaEventCreate(&e[1]));
  // every model's earlier work first, so the timed region holds only these steps
  for (mfdm_model* m : g->ms) MFDM_CU(cudaStreamSynchronize(m->stream));
  MFDM_CU(cudaEventRecord(e[0], g->stream));
  const int rc = group_run(g, nsteps);
  if (rc != MFDM_OK) return rc;
  MFDM_CU(cudaEventRecord(e[1], g->stream));
  MFDM_CU(cudaEventSynchronize(e[1]));
  MFDM_CU(cudaEventElapsedTime(total_ms, e[0], e[1]));
  return group_check(g);
}

int mfdm_group_close(mfdm_group* g) {
  group_destroy(g);
  return MFDM_OK;
}

int mfdm_set_field(mfdm_model* m, int field, const float* host) {
  if (!m || !host) return fail(MFDM_ERR_ARG, "null argument");
  float* p = nullptr;
  int rows = 0;
  int rc = field_ptr(m, field, &p, &rows);
  if (rc != MFDM_OK) return rc;
  DeviceGuard g(m->device);
  MFDM_CU(cudaMemcpy2DAsync(p, size_t(m->P) * sizeof(float), host, size_t(m->cfg.nx) * sizeof(float),
                            size_t(m->cfg.nx) * sizeof(float), size_t(rows), cudaMemcpyHostToDevice,
                            m->stream));
  MFDM_CU(cudaStreamSynchronize(m->stream));
  return MFDM_OK;
}

}  // extern "C"

// ---- adjoint-state gradients ---------------------------------------------------

namespace {

// Layout of one RK set, read off the handle's own buffers (set 0; the other
// sets are the same at a fixed stride).
mfdm::SetLayout set_layout(const mfdm_model* m) {
  mfdm::SetLayout L{};
  const Fields& S = m->S[0];
  const float* base = S.fvx;
  L.len = m->S[1].fvx - m->S[0].fvx;
  const float* arr[mfdm::kSetArrays] = {
      S.fvx, S.fvz, S.fp, S.svx, S.svz, S.ssx, S.ssz, S.ssxz,
      S.fx[0], S.fx[1], S.fx[2], S.fx[3], S.sx[0], S.sx[1], S.sx[2], S.sx[3],
      S.sz[0], S.sz[1], S.sz[2], S.sz[3], S.fz[0], S.fz[1], S.fz[2], S.fz[3]};
  const HostModel& h = m->cfg;
  const int npd = h.npd;
  for (int a = 0; a < mfdm::kSetArrays; ++a) {
    L.off[a] = arr[a] - base;
    if (a < 3) { L.rows[a] = h.nzf; L.pitch[a] = m->P; L.ncols[a] = h.nx; L.kind[a] = 0; }
    else if (a < 8) { L.rows[a] = h.nzs; L.pitch[a] = m->P; L.ncols[a] = h.nx; L.kind[a] = 1; }
    else if (a < 12) { L.rows[a] = npd > 0 ? h.nzf : 0; L.pitch[a] = m->Ps; L.ncols[a] = 2 * npd; L.kind[a] = 2; }
    else if (a < 16) { L.rows[a] = npd > 0 ? h.nzs : 0; L.pitch[a] = m->Ps; L.ncols[a] = 2 * npd; L.kind[a] = 3; }
    else if (a < 20) { L.rows[a] = npd; L.pitch[a] = m->P; L.ncols[a] = h.nx; L.kind[a] = 4; }
    else { L.rows[a] = m->C.cpml ? npd : 0; L.pitch[a] = m->P; L.ncols[a] = h.nx; L.kind[a] = 5; }
  }
  L.nx = h.nx; L.nzf = h.nzf; L.nzs = h.nzs; L.npd = npd;
  L.cpml = m->C.cpml;
  return L;
}

// The Fields view of a set-sized buffer.
Fields fields_at(const mfdm::SetLayout& L, float* base) {
  Fields F;
  float* p[mfdm::kSetArrays];
  for (int a = 0; a < mfdm::kSetArrays; ++a) p[a] = base + L.off[a];
  F.fvx = p[0]; F.fvz = p[1]; F.fp = p[2];
  F.svx = p[3]; F.svz = p[4]; F.ssx = p[5]; F.ssz = p[6]; F.ssxz = p[7];
  for (int q = 0; q < 4; ++q) {
    F.fx[q] = p[8 + q]; F.sx[q] = p[12 + q]; F.sz[q] = p[16 + q]; F.fz[q] = p[20 + q];
  }
  return F;
}

template <class T>
int dalloc(T** p, size_t n) {
  MFDM_CU(cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T)));
  return MFDM_OK;
}

// Assembles L_F^T and L_B^T by lattice probes of the stage kernel on the
// handle's own sets: input A (1 on the lattice points of one array), U^n = B
// (0), accumulator = Acc (scratch), output U = c k. Leaves the state at rest.
int adjoint_build(mfdm_model* m) {
  AdjointState* a = m->adj;
  const auto t0 = std::chrono::steady_clock::now();
  const mfdm::SetLayout& L = a->L;
  const long long n = L.len;
  cudaStream_t st = m->stream;
  int rc;
  if ((rc = clear_state(m)) != MFDM_OK) return rc;
  Coef C = m->C;
  C.srcx = -1;  // the operator without the source
  C.src_pos = nullptr;
  const int stage = 1;  // a middle stage: out = U^n + c k, with U^n = 0
  const float cc = C.rk_c[stage], scale = 1.0f / cc;
  mfdm::StageMaps maps;
  maps.fin = m->fst[1]; maps.sin = m->sst[1];
  maps.fun = m->fpw[2]; maps.sun = m->spw[2];
  maps.facc = m->fpw[3]; maps.sacc = m->spw[3];
  maps.fcoef = m->fco; maps.scoef = m->sco;
  const Fields &Out = m->S[0], &In = m->S[1], &Un = m->S[2], &Acc = m->S[3];
  // cells a stage updates: with input 0 and U^n = 1 the output is 1 exactly there
  MFDM_CU(mfdm::adj::fill(Un.fvx, n, 1.0f, st));
  MFDM_CU(mfdm::launch_stage(C, In, Out, Un, Acc, maps, stage, mfdm::kDirF, st));
  MFDM_CU(mfdm::adj::make_mask(Out.fvx, a->mask, n, st));
  MFDM_CU(cudaMemsetAsync(Un.fvx, 0, size_t(n) * sizeof(float), st));
  MFDM_CU(cudaMemsetAsync(Out.fvx, 0, size_t(n) * sizeof(float), st));
  unsigned long long* count = nullptr;
  int *cursor = nullptr, *err = nullptr;
  if ((rc = dalloc(&count, size_t(n) + 1)) != MFDM_OK) return rc;
  struct Free { void* p[3]; ~Free() { for (void* q : p) cudaFree(q); } } fr{{count, nullptr, nullptr}};
  if ((rc = dalloc(&cursor, size_t(n))) != MFDM_OK) return rc;
  fr.p[1] = cursor;
  if ((rc = dalloc(&err, 1)) != MFDM_OK) return rc;
  fr.p[2] = err;
  MFDM_CU(cudaMemsetAsync(err, 0, sizeof(int), st));
  for (int d = 0; d < 2; ++d) {
    mfdm::CsrT A;  // the full probed operator of this direction
    MFDM_CU(cudaMemsetAsync(count, 0, (size_t(n) + 1) * sizeof(unsigned long long), st));
    for (int pass = 0; pass < 2; ++pass) {
      if (pass == 1) {
        if ((rc = dalloc(&A.rowptr, size_t(n) + 1)) != MFDM_OK) return rc;
        MFDM_CU(mfdm::adj::scan(count, A.rowptr, n, &a->scan_tmp, &a->scan_bytes, st));
        MFDM_CU(cudaMemcpyAsync(&A.nnz, A.rowptr + n, sizeof(long long), cudaMemcpyDeviceToHost, st));
        MFDM_CU(cudaStreamSynchronize(st));
        if (A.nnz >= (1LL << 31) || n >= (1LL << 31))
          return fail(MFDM_ERR_ARG, "model too large for the adjoint operators");
        if ((rc = dalloc(&A.col, size_t(A.nnz))) != MFDM_OK) return rc;
        if ((rc = dalloc(&A.val, size_t(A.nnz))) != MFDM_OK) return rc;
        MFDM_CU(cudaMemsetAsync(cursor, 0, size_t(n) * sizeof(int), st));
      }
      for (int arr = 0; arr < mfdm::kSetArrays; ++arr) {
        if (L.rows[arr] <= 0) continue;
        for (int cz = 0; cz < 7; ++cz)
          for (int cx = 0; cx < 7; ++cx) {
            MFDM_CU(mfdm::adj::set_lattice(In.fvx, L, arr, cz, cx, 1.0f, st));
            MFDM_CU(mfdm::launch_stage(C, In, Out, Un, Acc, maps, stage, d, st));
            MFDM_CU(mfdm::adj::extract(Out.fvx, L, arr, cz, cx, scale, count,
                                       pass ? A.rowptr : nullptr, cursor, A.col, A.val, err, st));
            MFDM_CU(mfdm::adj::set_lattice(In.fvx, L, arr, cz, cx, 0.0f, st));
          }
      }
    }
    MFDM_CU(mfdm::adj::sort_rows(A, n, st));
    // keep only the non-interior outputs; the transposed interior stencil
    // covers the rest. Checked against the full operator on a random vector.
    mfdm::HybridT full;
    full.rest = A;
    mfdm::HybridT& H = a->H[d];
    H.qx = a->H[0].qx;
    H.qz = a->H[0].qz;
    cudaError_t e = mfdm::adj::drop_interior(A, L, &H.rest, count, &a->scan_tmp, &a->scan_bytes, st);
    if (e == cudaSuccess) e = mfdm::adj::list_rows(&H, L, count, &a->scan_tmp, &a->scan_bytes, st);
    float *x = a->mu, *y0 = a->kb[0], *y1 = a->kb[1];
    if (e == cudaSuccess) e = mfdm::adj::random_fill(x, n, 12345u + unsigned(d), st);
    if (e == cudaSuccess) e = mfdm::adj::apply_t(full, C, L, d, x, y0, st);
    if (e == cudaSuccess) e = mfdm::adj::apply_t(H, C, L, d, x, y1, st);
    cudaFree(A.rowptr);
    cudaFree(A.col);
    cudaFree(A.val);
    MFDM_CU(e);
    std::vector<float> h0(static_cast<size_t>(n)), h1(static_cast<size_t>(n));
    MFDM_CU(cudaMemcpyAsync(h0.data(), y0, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost, st));
    MFDM_CU(cudaMemcpyAsync(h1.data(), y1, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost, st));
    MFDM_CU(cudaStreamSynchronize(st));
    double num = 0.0, den = 0.0;
    for (size_t i = 0; i < h0.size(); ++i) {
      const double dd = double(h1[i]) - double(h0[i]);
      num += dd * dd;
      den += double(h0[i]) * double(h0[i]);
    }
    if (!(num <= 1e-8 * den))
      return fail(MFDM_ERR_CUDA, "adjoint operator assembly: the transposed interior stencil "
                                 "disagrees with the probed operator (relative L2 " +
                                     std::to_string(std::sqrt(num / std::max(den, 1e-300))) + ")");
  }
  int nerr = 0;
  MFDM_CU(cudaMemcpyAsync(&nerr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MFDM_CU(cudaStreamSynchronize(st));
  if (nerr) return fail(MFDM_ERR_CUDA, "adjoint operator assembly: " + std::to_string(nerr) +
                                           " outputs outside the 3-cell stencil radius");
  if ((rc = clear_state(m)) != MFDM_OK) return rc;
  if ((rc = rewind(m)) != MFDM_OK) return rc;
  a->built = true;
  a->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return MFDM_OK;
}

int ncp_of(int nsteps, int every) { return (nsteps + every - 1) / every; }

int adjoint_prepare(mfdm_model* m) {
  if (m->batch || m->nshots != 1)
    return fail(MFDM_ERR_ARG, "the adjoint runs on plain (single-shot) handles");
  if (!m->adj) {
    m->adj = new AdjointState();
    AdjointState* a = m->adj;
    a->L = set_layout(m);
    const size_t n = size_t(a->L.len);
    int rc;
    if ((rc = dalloc(&a->mask, n)) || (rc = dalloc(&a->lam, n)) || (rc = dalloc(&a->mu, n)) ||
        (rc = dalloc(&a->H[0].qx, n)) || (rc = dalloc(&a->H[0].qz, n)) ||
        (rc = dalloc(&a->kb[0], n)) || (rc = dalloc(&a->kb[1], n)) ||
        (rc = dalloc(&a->grad, size_t(2) * m->cfg.nzf * m->P + size_t(5) * m->cfg.nzs * m->P)))
      return rc;
    // Q fields off the interior set are never written and must stay 0
    MFDM_CU(cudaMemset(a->H[0].qx, 0, n * sizeof(float)));
    MFDM_CU(cudaMemset(a->H[0].qz, 0, n * sizeof(float)));
    int least = 0, greatest = 0;
    MFDM_CU(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    MFDM_CU(cudaStreamCreateWithPriority(&a->hi, cudaStreamNonBlocking, greatest));
    MFDM_CU(cudaStreamCreateWithPriority(&a->side_g, cudaStreamNonBlocking, least));
    MFDM_CU(cudaEventCreateWithFlags(&a->ev_enter, cudaEventDisableTiming));
    MFDM_CU(cudaEventCreateWithFlags(&a->ev_leave, cudaEventDisableTiming));
    for (cudaEvent_t& e : a->ev_seg) MFDM_CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (cudaEvent_t& e : a->ev_rev) MFDM_CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    MFDM_CU(cudaEventCreateWithFlags(&a->ev_kb, cudaEventDisableTiming));
    for (cudaEvent_t& e : a->ev_g) MFDM_CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  if (!m->adj->built) return adjoint_build(m);
  return MFDM_OK;
}

// dst[r][x] += float(grad[r][x]) over the seven gradient arrays stacked as rows
// (2 nz_f + 5 nz_s rows, device pitch P doubles, packed rows of nx floats).
__global__ void grad_accumulate_kernel(const double* __restrict__ g, int rows, int nx, int P,
                                       float* __restrict__ dst) {
  const size_t n = size_t(rows) * nx;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    const size_t r = i / nx, x = i - r * nx;
    dst[i] += float(g[r * P + x]);
  }
}

cudaError_t launch_grad_accumulate(const double* g, int rows, int nx, int P, float* dst,
                                   cudaStream_t st) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  grad_accumulate_kernel<<<unsigned(sms * 8), 256, 0, st>>>(g, rows, nx, P, dst);
  return cudaGetLastError();
}

double* grad_array(mfdm_model* m, int k) {
  const size_t nf = size_t(m->cfg.nzf) * m->P, ns = size_t(m->cfg.nzs) * m->P;
  return m->adj->grad + (k < 2 ? size_t(k) * nf : 2 * nf + size_t(k - 2) * ns);
}

// Encodes the TMA maps of the first `nslots` step slots of the slot buffer at
// `base` into `t` (once per buffer).
int slot_maps(mfdm_model* m, AdjointState::SlotTable& t, const float* base, size_t nslots) {
  if (t.base == base && t.maps.size() >= nslots) return MFDM_OK;
  const mfdm::SetLayout& L = m->adj->L;
  const size_t len = size_t(L.len);
  const int P = m->P, nzf = m->cfg.nzf, nzs = m->cfg.nzs;
  t.base = nullptr;
  t.maps.assign(nslots, AdjointState::SlotMaps{});
  int rc;
  for (size_t j = 0; j < nslots; ++j) {
    AdjointState::SlotMaps& M = t.maps[j];
    for (int s = 0; s < 4; ++s) {
      const float* set = base + (j * 4 + size_t(s)) * len;
      if ((rc = encode_block(&M.fst[s], set + L.off[0], P, nzf, 3, mfdm::kStageSW, true, m->nshots, m->region)) ||
          (rc = encode_block(&M.sst[s], set + L.off[3], P, nzs, 5, mfdm::kStageSW, true, m->nshots, m->region)))
        return rc;
    }
    const float* y1 = base + j * 4 * len;
    if ((rc = encode_block(&M.fun, y1 + L.off[0], P, nzf, 3, mfdm::kStageTX, false, m->nshots, m->region)) ||
        (rc = encode_block(&M.sun, y1 + L.off[3], P, nzs, 5, mfdm::kStageTX, false, m->nshots, m->region)))
      return rc;
  }
  t.base = base;
  return MFDM_OK;
}

// One step run in place in slot j of a slot buffer (maps `t`): stage 0 reads
// U^n from the slot's first set, stages 0-2 write the next three sets (the
// stage inputs the backward pass reads), the last stage writes U^{n+1} into the
// next slot's first set, or into the handle's state U after the run's last step.
int enqueue_slot_step(mfdm_model* m, int it, const AdjointState::SlotTable& t, size_t j,
                      bool last_of_run, cudaStream_t st) {
  AdjointState* a = m->adj;
  const mfdm::SetLayout& L = a->L;
  const size_t len = size_t(L.len);
  float* base = const_cast<float*>(t.base);
  const int d0 = (it & 1) ? mfdm::kDirB : mfdm::kDirF, d1 = 1 - d0;
  const int dir[4] = {d0, d1, d0, d1};
  Fields Y[4];
  for (int s = 0; s < 4; ++s) Y[s] = fields_at(L, base + (j * 4 + size_t(s)) * len);
  const Fields next = last_of_run ? m->S[0] : fields_at(L, base + (j + 1) * 4 * len);
  const AdjointState::SlotMaps& M = t.maps[j];
  const Fields& Acc = m->S[3];
  for (int s = 0; s < 4; ++s) {
    mfdm::StageMaps maps;
    maps.fin = M.fst[s];
    maps.sin = M.sst[s];
    maps.fun = M.fun;
    maps.sun = M.sun;
    maps.facc = m->fpw[3];
    maps.sacc = m->spw[3];
    maps.fcoef = m->fco;
    maps.scoef = m->sco;
    MFDM_CU(mfdm::launch_stage(m->C, Y[s], s < 3 ? Y[s + 1] : next, Y[0], Acc, maps, s, dir[s], st));
  }
  MFDM_CU(mfdm::launch_finish(m->C, next, st));
  return MFDM_OK;
}

// Transposed step n: lam holds lambda^{n+1} on entry and lambda^n on return;
// `slot` holds the step's four stage inputs.
int reverse_step(mfdm_model* m, int n, float* slot) {
  AdjointState* a = m->adj;
  const mfdm::SetLayout& L = a->L;
  const long long len = L.len;
  // the step runs on the high-priority stream (the caller orders it against
  // the handle's stream)
  cudaStream_t st = a->hi;
  const Coef& C = m->C;
  const int d0 = (n & 1) ? mfdm::kDirB : mfdm::kDirF, d1 = 1 - d0;
  Fields Y[4];
  for (int s = 0; s < 4; ++s) Y[s] = fields_at(L, slot + size_t(s) * size_t(len));
  double* g[7];
  for (int k = 0; k < 7; ++k) g[k] = grad_array(m, k);
  const float *c = C.rk_c, *w = C.rk_w;
  // mu = F^T lam and kb = c3 M mu: off the interface rows both were formed by
  // the previous transposed step's last stage (zero before the first); the
  // residuals of step n enter when n is a receiver sample
  const float* res = (n % m->gap == 0) ? a->res + size_t(n / m->gap) * 3 * size_t(m->cfg.nx) : nullptr;
  MFDM_CU(mfdm::adj::step_start(a->lam, L, C, res, a->mu, a->kb[0], a->mask, c[3], st));
  // Each stage: once kb[kin] is complete, its Q fields and sparse rows of L^T
  // kb (one launch) and the transposed product run on the main stream, and its
  // material-gradient accumulation on side_g. The product writes kb[1 - kin],
  // which the previous stage's gradient reads: it waits for that gradient
  // (ev_g[1 - kin]; a never-recorded event is no wait).
  auto stage = [&](int d, int sy, int kin, bool mask_lam, float ws, float cs, bool first) -> int {
    MFDM_CU(cudaEventRecord(a->ev_kb, st));
    MFDM_CU(mfdm::adj::prepare(a->H[d], C, L, a->kb[kin], st));
    MFDM_CU(cudaStreamWaitEvent(a->side_g, a->ev_kb, 0));
    MFDM_CU(mfdm::adj::gradient(C, L, Y[sy], a->kb[kin], g, d, nullptr, a->side_g));
    MFDM_CU(cudaEventRecord(a->ev_g[kin], a->side_g));
    MFDM_CU(cudaStreamWaitEvent(st, a->ev_g[1 - kin], 0));
    MFDM_CU(mfdm::adj::reverse_stage(a->H[d], C, L, d, a->kb[kin], a->lam, a->mask, mask_lam,
                                     a->kb[1 - kin], a->mu, ws, cs, true, first, st));
    return MFDM_OK;
  };
  int rc;
  // the first stage takes lam from mu (the step start leaves lam unfiltered)
  if ((rc = stage(d1, 3, 0, true, w[2], c[2], true)) != MFDM_OK) return rc;
  if ((rc = stage(d0, 2, 1, true, w[1], c[1], false)) != MFDM_OK) return rc;
  if ((rc = stage(d1, 1, 0, true, w[0], c[0], false)) != MFDM_OK) return rc;
  if ((rc = stage(d0, 0, 1, false, c[3], 0.f, false)) != MFDM_OK) return rc;
  // the step's stage inputs and kb are not reused before its last gradient ends
  MFDM_CU(cudaStreamWaitEvent(st, a->ev_g[1], 0));
  return MFDM_OK;
}

// Transposed steps u1-1 .. u0 with stage inputs at base (4 sets per step), on
// the high-priority stream. (Captured as a CUDA graph per segment shape the
// run measured 6 % slower: the chain's stream priorities over the gradient
// stream do not carry into graph nodes.)
int reverse_range(mfdm_model* m, int u0, int u1, float* base) {
  AdjointState* a = m->adj;
  const size_t len = size_t(a->L.len);
  for (int n = u1 - 1; n >= u0; --n) {
    const int rc = reverse_step(m, n, base + size_t(n - u0) * 4 * len);
    if (rc != MFDM_OK) return rc;
  }
  return MFDM_OK;
}

}  // namespace

extern "C" {

int mfdm_adjoint_set_memory(mfdm_model* m, long long bytes) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  if (bytes < 0) return fail(MFDM_ERR_ARG, "negative memory budget");
  DeviceGuard g(m->device);
  m->adj_keep_budget = bytes;
  if (m->adj) {
    if (bytes == 0) {
      MFDM_CU(cudaStreamSynchronize(m->stream));
      cudaFree(m->adj->keep);
      m->adj->keep = nullptr;
      m->adj->keep_floats = 0;
      m->adj->nkeep = 0;
    }
    m->adj->nsteps = -1;  // takes effect with the next mfdm_adjoint_forward
  }
  return MFDM_OK;
}

int mfdm_adjoint_set_inner(mfdm_model* m, int inner_every) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  if (inner_every < 0) return fail(MFDM_ERR_ARG, "negative inner checkpoint interval");
  m->adj_inner = inner_every;
  return MFDM_OK;
}

int mfdm_adjoint_forward(mfdm_model* m, int nsteps, int ckpt_every) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  if (nsteps < 1 || ckpt_every < 1) return fail(MFDM_ERR_ARG, "need nsteps >= 1 and ckpt_every >= 1");
  DeviceGuard g(m->device);
  int rc;
  if ((rc = adjoint_prepare(m)) != MFDM_OK) return rc;
  AdjointState* a = m->adj;
  const size_t len = size_t(a->L.len);
  const size_t ncp = size_t((nsteps + ckpt_every - 1) / ckpt_every);
  if (ncp > a->ckpt_sets) {
    cudaFree(a->ckpt);
    a->ckpt = nullptr;
    a->ckpt_sets = 0;
    if ((rc = dalloc(&a->ckpt, ncp * len)) != MFDM_OK) return rc;
    a->ckpt_sets = ncp;
  }
  // whole segments whose stage inputs fit the caller's memory budget are kept
  // now (the last ones, which the backward pass reaches first) and not recomputed
  const size_t seg_floats = size_t(ckpt_every) * 4 * len;
  const size_t nkeep = std::min(ncp, size_t(std::max<long long>(m->adj_keep_budget, 0)) /
                                         (seg_floats * sizeof(float)));
  if (nkeep * seg_floats > a->keep_floats) {
    cudaFree(a->keep);
    a->keep = nullptr;
    a->keep_floats = 0;
    if ((rc = dalloc(&a->keep, nkeep * seg_floats)) != MFDM_OK) return rc;
    a->keep_floats = nkeep * seg_floats;
    // cells a stage never writes (frozen rows and columns, ADE cells off the
    // strips) must read 0, as in the handle's own sets
    MFDM_CU(cudaMemset(a->keep, 0, nkeep * seg_floats * sizeof(float)));
  }
  if (nkeep > 0 && (rc = slot_maps(m, a->keep_tab, a->keep, nkeep * size_t(ckpt_every))) != MFDM_OK)
    return rc;
  a->nkeep = int(nkeep);
  a->nsteps = -1;
  if ((rc = clear_state(m)) != MFDM_OK) return rc;
  if ((rc = rewind(m)) != MFDM_OK) return rc;
  if ((rc = ensure_capacity(m, nsteps)) != MFDM_OK) return rc;
  for (size_t k = 0; k < ncp; ++k) {
    const int todo = std::min(ckpt_every, nsteps - int(k) * ckpt_every);
    if (k + nkeep >= ncp) {
      // kept: no checkpoint needed; the stages run in place in the keep buffer
      const size_t j0 = (k + nkeep - ncp) * size_t(ckpt_every);
      if (k + nkeep == ncp)  // the first kept step starts from the handle's state
        MFDM_CU(cudaMemcpyAsync(a->keep + j0 * 4 * len, m->S[0].fvx, len * sizeof(float),
                                cudaMemcpyDeviceToDevice, m->stream));
      for (int j = 0; j < todo; ++j) {
        const bool last = k + 1 == ncp && j + 1 == todo;
        if ((rc = enqueue_slot_step(m, m->host_step, a->keep_tab, j0 + size_t(j), last, m->stream)) !=
            MFDM_OK)
          return rc;
        ++m->host_step;
      }
    } else {
      MFDM_CU(cudaMemcpyAsync(a->ckpt + k * len, m->S[0].fvx, len * sizeof(float),
                              cudaMemcpyDeviceToDevice, m->stream));
      if ((rc = enqueue_steps(m, todo)) != MFDM_OK) return rc;
    }
  }
  MFDM_CU(cudaStreamSynchronize(m->stream));
  if ((rc = check_status(m)) != MFDM_OK) return rc;
  a->nsteps = nsteps;
  a->every = ckpt_every;
  return MFDM_OK;
}

int mfdm_adjoint_backward(mfdm_model* m, const float* res_svx, const float* res_svz,
                          const float* res_fp, mfdm_coef_grad* out) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  AdjointState* a = m->adj;
  if (!a || a->nsteps < 1 || m->host_step != a->nsteps)
    return fail(MFDM_ERR_ARG, "mfdm_adjoint_backward needs the mfdm_adjoint_forward run just before it");
  DeviceGuard g(m->device);
  int rc;
  const int nsteps = a->nsteps, every = a->every, nx = m->cfg.nx;
  const size_t len = size_t(a->L.len);
  const int ns = (nsteps + m->gap - 1) / m->gap;
  // residuals, [ns][3][nx] in the receiver-buffer order (svx, svz, fp)
  const size_t rf = size_t(ns) * 3 * nx;
  if (rf > a->res_floats) {
    cudaFree(a->res);
    a->res = nullptr;
    a->res_floats = 0;
    if ((rc = dalloc(&a->res, rf)) != MFDM_OK) return rc;
    a->res_floats = rf;
  }
  {
    std::vector<float> h(rf, 0.f);
    const float* src[3] = {res_svx, res_svz, res_fp};
    for (int j = 0; j < ns; ++j)
      for (int q = 0; q < 3; ++q)
        if (src[q]) std::memcpy(&h[(size_t(j) * 3 + q) * nx], src[q] + size_t(j) * nx, nx * sizeof(float));
    MFDM_CU(cudaMemcpy(a->res, h.data(), rf * sizeof(float), cudaMemcpyHostToDevice));
  }
  const int ncp = ncp_of(nsteps, every);
  // second level: a recomputed segment first re-runs keeping a state every
  // `inner` steps, then recomputes and reverses one inner stretch at a time
  const int inner = (m->adj_inner > 0 && m->adj_inner < every) ? m->adj_inner : every;
  const size_t ninner = size_t((every + inner - 1) / inner);
  if (a->nkeep < ncp && size_t(inner) > a->seg_steps) {
    cudaFree(a->seg);
    cudaFree(a->seg2);  // re-made at the new size when the overlap uses it
    a->seg = nullptr;
    a->seg2 = nullptr;
    a->seg_steps = 0;
    if ((rc = dalloc(&a->seg, size_t(inner) * 4 * len)) != MFDM_OK) return rc;
    // cells a stage never writes must read 0, as in the handle's own sets
    MFDM_CU(cudaMemset(a->seg, 0, size_t(inner) * 4 * len * sizeof(float)));
    a->seg_steps = size_t(inner);
  }
  if (a->nkeep < ncp && (rc = slot_maps(m, a->seg_tab[0], a->seg, a->seg_steps)) != MFDM_OK)
    return rc;
  if (a->nkeep < ncp && inner < every && ninner > a->inner_sets) {
    cudaFree(a->inner);
    a->inner = nullptr;
    a->inner_sets = 0;
    if ((rc = dalloc(&a->inner, ninner * len)) != MFDM_OK) return rc;
    a->inner_sets = ninner;
  }
  cudaStream_t st = m->stream;
  const size_t gbytes = (size_t(2) * m->cfg.nzf * m->P + size_t(5) * m->cfg.nzs * m->P) * sizeof(double);
  a->grad_ready = false;
  MFDM_CU(cudaMemsetAsync(a->grad, 0, gbytes, st));
  MFDM_CU(cudaMemsetAsync(a->lam, 0, len * sizeof(float), st));
  MFDM_CU(cudaMemsetAsync(a->mu, 0, len * sizeof(float), st));
  MFDM_CU(cudaMemsetAsync(a->kb[0], 0, len * sizeof(float), st));
  a->nsteps = -1;
  // The reverse steps run on a->hi (high priority); the handle's stream `st`
  // restores checkpoints and recomputes segments. With a second stage-input
  // buffer, segment k-1 is recomputed into it while segment k is reversed.
  cudaStream_t hi = a->hi;
  MFDM_CU(cudaEventRecord(a->ev_enter, st));  // the reverse chain starts after the memsets
  MFDM_CU(cudaStreamWaitEvent(hi, a->ev_enter, 0));
  bool dbl = inner == every && a->nkeep < ncp - 1;
  if (dbl && a->seg2 == nullptr) {
    if (cudaMalloc(&a->seg2, a->seg_steps * 4 * len * sizeof(float)) != cudaSuccess) {
      (void)cudaGetLastError();  // not enough memory for two: one buffer, no overlap
      a->seg2 = nullptr;
      dbl = false;
    } else {
      MFDM_CU(cudaMemset(a->seg2, 0, a->seg_steps * 4 * len * sizeof(float)));
    }
  }
  if (dbl && (rc = slot_maps(m, a->seg_tab[1], a->seg2, a->seg_steps)) != MFDM_OK) return rc;
  auto buf_of = [&](int k) { return (dbl && (k & 1)) ? 1 : 0; };
  auto buf_ptr = [&](int b) { return b ? a->seg2 : a->seg; };
  // restore checkpoint k into the first slot of buffer b and recompute steps
  // u0..u1-1 in place in its slots (after the last reverse that read it)
  auto recompute = [&](int k, int u0, int u1, int b, bool from_ckpt, const float* from) -> int {
    MFDM_CU(cudaStreamWaitEvent(st, a->ev_rev[b], 0));
    MFDM_CU(cudaMemcpyAsync(buf_ptr(b), from_ckpt ? a->ckpt + size_t(k) * len : from,
                            len * sizeof(float), cudaMemcpyDeviceToDevice, st));
    MFDM_CU(mfdm::launch_set_step(m->C, u0, st));
    for (int n = u0; n < u1; ++n) {
      int rc2;
      if ((rc2 = enqueue_slot_step(m, n, a->seg_tab[b], size_t(n - u0), n + 1 == u1, st)) != MFDM_OK)
        return rc2;
    }
    MFDM_CU(cudaEventRecord(a->ev_seg[b], st));
    return MFDM_OK;
  };
  // reverse steps u1-1..u0 from buffer b, once their recompute is done
  auto reverse = [&](int u0, int u1, int b) -> int {
    MFDM_CU(cudaStreamWaitEvent(hi, a->ev_seg[b], 0));
    int rc2;
    if ((rc2 = reverse_range(m, u0, u1, buf_ptr(b))) != MFDM_OK) return rc2;
    MFDM_CU(cudaEventRecord(a->ev_rev[b], hi));
    return MFDM_OK;
  };
  int prepared = -1;  // the segment already recomputed ahead
  for (int k = ncp - 1; k >= 0; --k) {
    const int t0 = k * every, t1 = std::min(nsteps, t0 + every);
    if (k + a->nkeep >= ncp) {
      // kept by the forward pass
      float* base = a->keep + size_t(k + a->nkeep - ncp) * size_t(every) * 4 * len;
      if ((rc = reverse_range(m, t0, t1, base)) != MFDM_OK) return rc;
      continue;
    }
    if (inner < every) {
      // re-run the segment keeping a state every `inner` steps (after the
      // last reverse, whose stretch of the segment buffer it overwrites)
      MFDM_CU(cudaStreamWaitEvent(st, a->ev_rev[0], 0));
      MFDM_CU(cudaMemcpyAsync(m->S[0].fvx, a->ckpt + size_t(k) * len, len * sizeof(float),
                              cudaMemcpyDeviceToDevice, st));
      MFDM_CU(mfdm::launch_set_step(m->C, t0, st));
      m->host_step = t0;
      for (int i = 0; t0 + i * inner < t1; ++i) {
        MFDM_CU(cudaMemcpyAsync(a->inner + size_t(i) * len, m->S[0].fvx, len * sizeof(float),
                                cudaMemcpyDeviceToDevice, st));
        const int todo = std::min(inner, t1 - (t0 + i * inner));
        if (t0 + (i + 1) * inner < t1 && (rc = enqueue_steps(m, todo)) != MFDM_OK) return rc;
      }
      for (int i = (t1 - t0 - 1) / inner; i >= 0; --i) {
        const int u0 = t0 + i * inner, u1 = std::min(t1, u0 + inner);
        if ((rc = recompute(k, u0, u1, 0, false, a->inner + size_t(i) * len)) != MFDM_OK) return rc;
        if ((rc = reverse(u0, u1, 0)) != MFDM_OK) return rc;
      }
      continue;
    }
    if (prepared != k && (rc = recompute(k, t0, t1, buf_of(k), true, nullptr)) != MFDM_OK) return rc;
    if (dbl && k > 0) {  // the next segment to reverse, recomputed meanwhile
      const int p0 = (k - 1) * every, p1 = std::min(nsteps, p0 + every);
      if ((rc = recompute(k - 1, p0, p1, buf_of(k - 1), true, nullptr)) != MFDM_OK) return rc;
      prepared = k - 1;
    }
    if ((rc = reverse(t0, t1, buf_of(k))) != MFDM_OK) return rc;
  }
  MFDM_CU(cudaEventRecord(a->ev_leave, hi));
  MFDM_CU(cudaStreamWaitEvent(st, a->ev_leave, 0));
  MFDM_CU(cudaStreamSynchronize(st));
  if (out) {
    double* dst[7] = {out->K, out->rcp_rho_f, out->C11, out->C13, out->C33, out->C55, out->rcp_rho_s};
    for (int k = 0; k < 7; ++k) {
      if (!dst[k]) continue;
      const int rows = k < 2 ? m->cfg.nzf : m->cfg.nzs;
      MFDM_CU(cudaMemcpy2D(dst[k], size_t(nx) * sizeof(double), grad_array(m, k),
                           size_t(m->P) * sizeof(double), size_t(nx) * sizeof(double), size_t(rows),
                           cudaMemcpyDeviceToHost));
    }
  }
  // the recomputation left a mid-run state: back to rest
  if ((rc = clear_state(m)) != MFDM_OK) return rc;
  if ((rc = rewind(m)) != MFDM_OK) return rc;
  m->adj->grad_ready = true;
  return check_status(m);
}

int mfdm_adjoint_accumulate_grad_f32(mfdm_model* m, float* dst, void* stream) {
  if (!m || !dst) return fail(MFDM_ERR_ARG, "null argument");
  if (!m->adj || !m->adj->grad || !m->adj->grad_ready)
    return fail(MFDM_ERR_ARG, "no gradient: call mfdm_adjoint_backward first");
  DeviceGuard g(m->device);
  const int rows = 2 * m->cfg.nzf + 5 * m->cfg.nzs;
  MFDM_CU(launch_grad_accumulate(m->adj->grad, rows, m->cfg.nx, m->P, dst,
                                 static_cast<cudaStream_t>(stream)));
  return MFDM_OK;
}

}  // extern "C"

// ---- solid only with a free surface (PmlFs::SolidOnly) -------------------------

struct mfdm_solid {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nx = 0, nz = 0, npd = 0, P = 0, Ps = 0;
  float dt = 0.f, fpeak = 0.f;
  int nt = 0, snapshot = 1, gap = 1;
  std::vector<int> srcx, srcz;
  int isrc = 0, host_step = 0;
  char* dmem = nullptr;
  size_t dbytes = 0;
  mfdm::solid::SFields S[4];  // U, stage A, stage B, accumulator
  mfdm::solid::SCoef C{};
  float* d_src = nullptr;
  int src_steps = 0;
  float* d_rec = nullptr;
  int rec_cap = 0;
  HostModel pml;  // PML scalars and the time step for the table builders
  cudaGraphExec_t graph = nullptr;
};

namespace {

// The arrays of one solid-only model, [nz][nx], in the caller's memory or in `own`.
struct SolidHost {
  int nx = 0, nz = 0;
  HostModel p;  // scalars: npd, npow, thickness, vp_max, rc, beta0, fpeak, dt, nt, snapshot, sources
  std::vector<float> own[10];
  const float* a[10] = {};  // C11, C13, C33, C55, rho, J, xi_x, xi_z, ze_x, ze_z
};

// Reads a calc_type 0 JSON (src/elements.cu:64-176 with the solid-only branches).
int load_json_solid(const char* path, SolidHost& h) {
  try {
    const mfdm::JsonConfig J = mfdm::JsonConfig::from_file(path);
    HostModel& p = h.p;
    p.fpeak = J.get_float("base.fpeak");
    p.dt = J.get_float("base.dt");
    p.nt = J.get_int("base.nt");
    p.snapshot = J.get_int("base.snapshot");
    const int bdy = J.get_int("grid.boundary_type");
    if (J.get_int("grid.calc_type") != 0 || (bdy != 1 && bdy != 2))
      return fail(MFDM_ERR_ARG,
                  "unsupported configuration: solid-only runs need calc_type 0 with "
                  "boundary_type 2 (free surface on top, CFS-PML sides and bottom) or 1 "
                  "(CFS-PML on all four sides)");
    p.bdy = bdy;
    const size_t nsrc = J.size("grid.src_pos.posx");
    for (size_t i = 0; i < nsrc; ++i) {
      p.srcx.push_back(J.get_int("grid.src_pos.posx", i));
      p.srcz.push_back(J.get_int("grid.src_pos.posz", i));
    }
    h.nx = J.get_int("grid.solid.nx");
    h.nz = J.get_int("grid.solid.nz");
    p.npd = J.get_int("PML.npd");
    p.thickness = J.get_float("PML.thickness");
    p.npow = J.get_int("PML.NPOW");
    p.vp_max = J.get_float("PML.Vp_max");
    p.rc = J.get_float("PML.Rc");
    p.beta0 = J.get_float("PML.beta0");
    if (h.nx <= 0 || h.nz <= 0) return fail(MFDM_ERR_CONFIG, "bad grid size");
    const size_t n = size_t(h.nx) * h.nz;
    const char* keys[10] = {"grid.solid.C11", "grid.solid.C13", "grid.solid.C33",
                            "grid.solid.C55", "grid.solid.rho", "grid.jacob.J",
                            "grid.jacob.xi_x", "grid.jacob.xi_z", "grid.jacob.ze_x",
                            "grid.jacob.ze_z"};
    for (int k = 0; k < 10; ++k) {
      const int rc = read_bin(J.get_string(keys[k]), n, h.own[k]);
      if (rc != MFDM_OK) return rc;
      h.a[k] = h.own[k].data();
    }
  } catch (const std::exception& e) {
    return fail(MFDM_ERR_CONFIG, e.what());
  }
  return MFDM_OK;
}

int json_calc_type(const char* path, int* calc_type) {
  try {
    *calc_type = mfdm::JsonConfig::from_file(path).get_int("grid.calc_type");
  } catch (const std::exception& e) {
    return fail(MFDM_ERR_CONFIG, e.what());
  }
  return MFDM_OK;
}

void solid_release_graph(mfdm_solid* m) {
  if (m->graph) {
    cudaGraphExecDestroy(m->graph);
    m->graph = nullptr;
  }
}

void solid_destroy(mfdm_solid* m) {
  if (!m) return;
  DeviceGuard g(m->device);
  solid_release_graph(m);
  if (m->stream) cudaStreamSynchronize(m->stream);
  if (m->d_src) cudaFree(m->d_src);
  if (m->d_rec) cudaFree(m->d_rec);
  if (m->dmem) cudaFree(m->dmem);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

int solid_capacity(mfdm_solid* m, int steps) {
  if (steps > m->src_steps) {
    const int cap = std::max(steps, m->src_steps * 2);
    std::vector<float> amp(size_t(cap) * 4);
    fill_src_table(m->pml, m->fpeak, cap, amp.data());
    float* d = nullptr;
    MFDM_CU(cudaMalloc(&d, amp.size() * sizeof(float)));
    MFDM_CU(cudaMemcpy(d, amp.data(), amp.size() * sizeof(float), cudaMemcpyHostToDevice));
    if (m->d_src) cudaFree(m->d_src);
    m->d_src = d;
    m->src_steps = cap;
    solid_release_graph(m);
  }
  const int need = (steps + m->gap - 1) / m->gap;
  if (need > m->rec_cap) {
    const int cap = std::max(need, m->rec_cap * 2);
    float* d = nullptr;
    MFDM_CU(cudaMalloc(&d, size_t(cap) * m->nx * sizeof(float)));
    MFDM_CU(cudaMemset(d, 0, size_t(cap) * m->nx * sizeof(float)));
    if (m->d_rec) {
      MFDM_CU(cudaMemcpy(d, m->d_rec, size_t(m->rec_cap) * m->nx * sizeof(float),
                         cudaMemcpyDeviceToDevice));
      cudaFree(m->d_rec);
    }
    m->d_rec = d;
    m->rec_cap = cap;
    solid_release_graph(m);
  }
  m->C.src_amp = m->d_src;
  m->C.src_steps = m->src_steps;
  m->C.rec = m->d_rec;
  m->C.rec_cap = m->rec_cap;
  return MFDM_OK;
}

int solid_enqueue_step(mfdm_solid* m, int it, cudaStream_t st) {
  const int d0 = (it & 1) ? mfdm::kDirB : mfdm::kDirF, d1 = 1 - d0;
  const mfdm::solid::SFields &U = m->S[0], &A = m->S[1], &B = m->S[2], &Acc = m->S[3];
  const mfdm::solid::SFields* in[4] = {&U, &A, &B, &A};
  const mfdm::solid::SFields* out[4] = {&A, &B, &A, &U};
  const int dir[4] = {d0, d1, d0, d1};
  for (int s = 0; s < 4; ++s)
    MFDM_CU(mfdm::solid::launch_stage(m->C, *in[s], *out[s], U, Acc, s, dir[s], st));
  MFDM_CU(mfdm::solid::launch_finish(m->C, U, st));
  return MFDM_OK;
}

int solid_enqueue_steps(mfdm_solid* m, int nsteps) {
  int rc;
  while (nsteps > 0) {
    if ((m->host_step & 1) == 0 && nsteps >= kGraphSteps) {
      if (!m->graph) {
        cudaGraph_t g = nullptr;
        MFDM_CU(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
        rc = MFDM_OK;
        for (int k = 0; k < kGraphSteps && rc == MFDM_OK; ++k) rc = solid_enqueue_step(m, k, m->stream);
        const cudaError_t e = cudaStreamEndCapture(m->stream, &g);
        if (rc != MFDM_OK) {
          if (g) cudaGraphDestroy(g);
          return rc;
        }
        if (e != cudaSuccess) return fail(MFDM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        const cudaError_t e2 = cudaGraphInstantiate(&m->graph, g, 0);
        cudaGraphDestroy(g);
        if (e2 != cudaSuccess)
          return fail(MFDM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2));
      }
      MFDM_CU(cudaGraphLaunch(m->graph, m->stream));
      m->host_step += kGraphSteps;
      nsteps -= kGraphSteps;
    } else {
      if ((rc = solid_enqueue_step(m, m->host_step, m->stream)) != MFDM_OK) return rc;
      ++m->host_step;
      --nsteps;
    }
  }
  return MFDM_OK;
}

int solid_rewind(mfdm_solid* m, bool clear) {
  const size_t set_bytes = size_t(reinterpret_cast<char*>(m->S[1].vx) - reinterpret_cast<char*>(m->S[0].vx));
  if (clear) MFDM_CU(cudaMemsetAsync(m->S[0].vx, 0, 4 * set_bytes, m->stream));
  if (m->d_rec)
    MFDM_CU(cudaMemsetAsync(m->d_rec, 0, size_t(m->rec_cap) * m->nx * sizeof(float), m->stream));
  MFDM_CU(cudaMemsetAsync(m->C.status, 0, sizeof(int), m->stream));
  m->host_step = 0;
  MFDM_CU(mfdm::solid::launch_set_step(m->C, 0, m->stream));
  MFDM_CU(cudaStreamSynchronize(m->stream));
  return MFDM_OK;
}

int solid_build(mfdm_solid* m, const SolidHost& h, int device) {
  const HostModel& p = h.p;
  if (h.nx < 8 || h.nz < 8) return fail(MFDM_ERR_ARG, "grid too small: need nx, nz >= 8");
  if (p.npd < 0 || 2 * p.npd > h.nx - 6 || p.npd + 7 > h.nz)
    return fail(MFDM_ERR_ARG, "PML width npd does not fit the grid");
  const bool cpml = p.bdy == 1;
  if (cpml && 2 * p.npd + 6 > h.nz)
    return fail(MFDM_ERR_ARG, "the top and bottom PML bands overlap: need nz >= 2 npd + 6");
  if (cpml && h.nz < 34)
    return fail(MFDM_ERR_ARG, "CFS-PML on four sides records row 30: need nz >= 34");
  if (!(p.dt > 0.f) || !(p.fpeak > 0.f)) return fail(MFDM_ERR_ARG, "dt and fpeak must be > 0");
  if (p.snapshot < 1 || p.nt < 0) return fail(MFDM_ERR_ARG, "need snapshot >= 1 and nt >= 0");
  for (size_t i = 0; i < p.srcx.size(); ++i)
    if (p.srcx[i] < 0 || p.srcx[i] >= h.nx || p.srcz[i] < 0 || p.srcz[i] >= h.nz)
      return fail(MFDM_ERR_ARG, "source outside the grid");
  m->device = device;
  int ndev = 0;
  MFDM_CU(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(MFDM_ERR_ARG, "no such CUDA device");
  MFDM_CU(cudaSetDevice(device));
  MFDM_CU(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  const int nx = h.nx, nz = h.nz, npd = p.npd;
  m->nx = nx; m->nz = nz; m->npd = npd;
  m->dt = p.dt; m->fpeak = p.fpeak; m->nt = p.nt; m->snapshot = p.snapshot;
  m->gap = std::max(1, int(1e-3 / double(p.dt) + 0.5));  // src/main.cu:92
  m->srcx = p.srcx; m->srcz = p.srcz;
  m->pml = p;
  const int P = round_up(nx, 32), Ps = round_up(std::max(2 * npd, 1), 4), npdr = std::max(npd, 1);
  m->P = P; m->Ps = Ps;
  size_t off = 0;
  auto take = [&](size_t nfloats) {
    const size_t o = off;
    off += (nfloats * sizeof(float) + 255) / 256 * 256;
    return o;
  };
  const size_t n = size_t(nz) * P;
  size_t o_arr[10];
  for (int k = 0; k < 10; ++k) o_arr[k] = take(n);
  const size_t o_alm = take(size_t(6) * P), o_px = take(size_t(nx) * 4), o_pz = take(size_t(nz) * 4),
               o_misc = take(64);
  size_t o_set[4];
  const int zrows = cpml ? 2 * npdr : npdr;  // zeta-ADE rows: bottom band (+ top band)
  for (int s = 0; s < 4; ++s) {
    o_set[s] = take(5 * n);
    for (int q = 0; q < 4; ++q) take(size_t(nz) * Ps);
    for (int q = 0; q < 4; ++q) take(size_t(zrows) * P);
  }
  const size_t set_floats = (o_set[1] - o_set[0]) / sizeof(float);
  m->dbytes = off;
  MFDM_CU(cudaMalloc(&m->dmem, off));
  MFDM_CU(cudaMemsetAsync(m->dmem, 0, off, m->stream));
  char* base = m->dmem;
  auto F = [&](size_t o) { return reinterpret_cast<float*>(base + o); };
  for (int s = 0; s < 4; ++s) {
    mfdm::solid::SFields& S = m->S[s];
    float* b = F(o_set[s]);
    S.vx = b; S.vz = b + n; S.sx = b + 2 * n; S.sz = b + 3 * n; S.sxz = b + 4 * n;
    size_t o = (5 * n * sizeof(float) + 255) / 256 * 256;
    for (int q = 0; q < 4; ++q) {
      S.x[q] = reinterpret_cast<float*>(reinterpret_cast<char*>(b) + o);
      o += (size_t(nz) * Ps * sizeof(float) + 255) / 256 * 256;
    }
    for (int q = 0; q < 4; ++q) {
      S.z[q] = reinterpret_cast<float*>(reinterpret_cast<char*>(b) + o);
      o += (size_t(zrows) * P * sizeof(float) + 255) / 256 * 256;
    }
    if (o / sizeof(float) > set_floats) return fail(MFDM_ERR_ARG, "internal layout error");
  }
  mfdm::solid::SCoef& C = m->C;
  C.nx = nx; C.nz = nz; C.P = P; C.Ps = Ps; C.npd = npd;
  C.cpml = cpml ? 1 : 0;
  C.rec_row = cpml ? 30 : 3;  // src/main.cu:303-311
  // the density slot holds 1/rho (FP64 reciprocal rounded once): the momentum
  // right-hand side multiplies instead of dividing
  std::vector<float> rcp_rho(size_t(nx) * nz);
  for (size_t k = 0; k < rcp_rho.size(); ++k) rcp_rho[k] = float(1.0 / double(h.a[4][k]));
  const float* arr[10];
  for (int k = 0; k < 10; ++k) {
    arr[k] = F(o_arr[k]);
    MFDM_CU(cudaMemcpy2DAsync(F(o_arr[k]), size_t(P) * sizeof(float), k == 4 ? rcp_rho.data() : h.a[k],
                              size_t(nx) * sizeof(float), size_t(nx) * sizeof(float), size_t(nz),
                              cudaMemcpyHostToDevice, m->stream));
  }
  C.C11 = arr[0]; C.C13 = arr[1]; C.C33 = arr[2]; C.C55 = arr[3]; C.rcp_rho = arr[4];
  C.J = arr[5]; C.xix = arr[6]; C.xiz = arr[7]; C.zex = arr[8]; C.zez = arr[9];
  // ALM coefficients of the free-surface row, in double from the model's floats
  // (src/elements.cu:907-977)
  std::vector<float> alm(size_t(6) * P, 0.f);
  for (int ix = 0; ix < nx; ++ix) {
    const size_t i = size_t(3) * nx + ix;
    const double xi_x = h.a[6][i], xi_z = h.a[7][i], ze_x = h.a[8][i], ze_z = h.a[9][i];
    const double c11 = h.a[0][i], c13 = h.a[1][i], c33 = h.a[2][i], c55 = h.a[3][i];
    const double Dz11 = c11 * ze_x * ze_x + c55 * ze_z * ze_z;
    const double Dz12 = (c13 + c55) * ze_x * ze_z;
    const double Dz22 = c55 * ze_x * ze_x + c33 * ze_z * ze_z;
    const double Dx11 = c11 * ze_x * xi_x + c55 * ze_z * xi_z;
    const double Dx12 = c13 * ze_x * xi_z + c55 * ze_z * xi_x;
    const double Dx21 = c13 * ze_z * xi_x + c55 * ze_x * xi_z;
    const double Dx22 = c55 * ze_x * xi_x + c33 * ze_z * xi_z;
    const double det = Dz11 * Dz22 - Dz12 * Dz12;
    double m11 = 0, m12 = 0, m21 = 0, m22 = 0;
    if (std::abs(det) >= 1e-14) {
      const double i11 = Dz22 / det, i12 = -Dz12 / det, i22 = Dz11 / det;
      m11 = i11 * Dx11 + i12 * Dx21;
      m12 = i11 * Dx12 + i12 * Dx22;
      m21 = i12 * Dx11 + i22 * Dx21;
      m22 = i12 * Dx12 + i22 * Dx22;
    }
    alm[0 * size_t(P) + ix] = float(xi_x - ze_x * m11);
    alm[1 * size_t(P) + ix] = float(-ze_z * m21);
    alm[2 * size_t(P) + ix] = float(xi_z - ze_z * m11 - ze_x * m21);
    alm[3 * size_t(P) + ix] = float(-ze_x * m12);
    alm[4 * size_t(P) + ix] = float(xi_z - ze_z * m22);
    alm[5 * size_t(P) + ix] = float(xi_x - ze_z * m12 - ze_x * m22);
  }
  MFDM_CU(cudaMemcpyAsync(F(o_alm), alm.data(), alm.size() * sizeof(float), cudaMemcpyHostToDevice, m->stream));
  C.alm = F(o_alm);
  std::vector<float4> px, pz;
  pml_profile(p, nx, true, true, p.fpeak, p.beta0, px);
  pml_profile(p, nz, cpml, true, p.fpeak, p.beta0, pz);  // top band only without a free surface
  MFDM_CU(cudaMemcpyAsync(F(o_px), px.data(), px.size() * sizeof(float4), cudaMemcpyHostToDevice, m->stream));
  MFDM_CU(cudaMemcpyAsync(F(o_pz), pz.data(), pz.size() * sizeof(float4), cudaMemcpyHostToDevice, m->stream));
  C.pmlx = reinterpret_cast<const float4*>(F(o_px));
  C.pmlz = reinterpret_cast<const float4*>(F(o_pz));
  int* misc = reinterpret_cast<int*>(F(o_misc));
  C.step = misc;
  C.done = reinterpret_cast<unsigned*>(misc + 1);
  C.status = misc + 2;
  // RK4 weights formed in float like the reference (src/pml_fs_kernels.cu:95-380)
  const float dt = p.dt;
  C.rk_c[0] = dt / 2; C.rk_c[1] = dt / 2; C.rk_c[2] = dt; C.rk_c[3] = dt / 6;
  C.rk_w[0] = dt / 6; C.rk_w[1] = dt / 3; C.rk_w[2] = dt / 3;
  C.gap = m->gap;
  C.srcx = m->srcx.empty() ? -1 : m->srcx[0];
  C.srcz = m->srcx.empty() ? 0 : m->srcz[0];
  int rc;
  if ((rc = solid_capacity(m, std::max(p.nt, 1))) != MFDM_OK) return rc;
  MFDM_CU(cudaStreamSynchronize(m->stream));
  return solid_rewind(m, false);
}

int solid_open(SolidHost&& h, int device, mfdm_solid** out) {
  if (!out) return fail(MFDM_ERR_ARG, "null output handle");
  *out = nullptr;
  int prev = -1;
  cudaGetDevice(&prev);
  mfdm_solid* m = new mfdm_solid();
  const int rc = solid_build(m, h, device);
  if (prev >= 0) cudaSetDevice(prev);
  if (rc != MFDM_OK) {
    const std::string msg = g_err;
    solid_destroy(m);
    g_err = msg;
    return rc;
  }
  *out = m;
  return MFDM_OK;
}

int solid_field_ptr(mfdm_solid* m, int field, float** p) {
  const mfdm::solid::SFields& U = m->S[0];
  switch (field) {
    case MFDM_SOLID_VX: *p = U.vx; break;
    case MFDM_SOLID_VZ: *p = U.vz; break;
    case MFDM_SOLID_SX: *p = U.sx; break;
    case MFDM_SOLID_SZ: *p = U.sz; break;
    case MFDM_SOLID_SXZ: *p = U.sxz; break;
    default: return fail(MFDM_ERR_ARG, "a solid-only model has only the solid fields");
  }
  return MFDM_OK;
}

}  // namespace

extern "C" {

int mfdm_solid_open_json(const char* json_path, int device, mfdm_solid** out) {
  if (!json_path) return fail(MFDM_ERR_ARG, "null JSON path");
  SolidHost h;
  const int rc = load_json_solid(json_path, h);
  if (rc != MFDM_OK) return rc;
  return solid_open(std::move(h), device, out);
}

int mfdm_solid_open_desc(const mfdm_solid_desc* d, int device, mfdm_solid** out) {
  if (!d) return fail(MFDM_ERR_ARG, "null descriptor");
  SolidHost h;
  h.nx = d->nx; h.nz = d->nz;
  HostModel& p = h.p;
  p.fpeak = d->fpeak; p.dt = d->dt; p.nt = d->nt; p.snapshot = d->snapshot;
  p.npd = d->npd; p.npow = d->npow; p.thickness = d->thickness; p.vp_max = d->vp_max;
  p.rc = d->rc; p.beta0 = d->beta0;
  p.bdy = d->boundary_type == 1 ? 1 : 2;
  for (int i = 0; i < d->nsrc; ++i) {
    if (!d->src_x || !d->src_z) return fail(MFDM_ERR_ARG, "null source arrays");
    p.srcx.push_back(d->src_x[i]);
    p.srcz.push_back(d->src_z[i]);
  }
  const float* a[10] = {d->C11, d->C13, d->C33, d->C55, d->rho, d->J, d->xi_x, d->xi_z, d->ze_x, d->ze_z};
  for (int k = 0; k < 10; ++k) {
    if (!a[k]) return fail(MFDM_ERR_ARG, "null model array");
    h.a[k] = a[k];
  }
  return solid_open(std::move(h), device, out);
}

int mfdm_solid_set_shot(mfdm_solid* m, int isrc, int reset_state) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  if (isrc < 0 || (isrc >= int(m->srcx.size()) && !m->srcx.empty()))
    return fail(MFDM_ERR_ARG, "shot index out of range");
  DeviceGuard g(m->device);
  m->isrc = isrc;
  m->C.srcx = m->srcx.empty() ? -1 : m->srcx[size_t(isrc)];
  m->C.srcz = m->srcx.empty() ? 0 : m->srcz[size_t(isrc)];
  solid_release_graph(m);  // the source cell is baked into the kernel arguments
  return solid_rewind(m, reset_state != 0);
}

int mfdm_solid_step(mfdm_solid* m, int nsteps) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  if (nsteps < 0) return fail(MFDM_ERR_ARG, "negative step count");
  DeviceGuard g(m->device);
  int rc;
  if ((rc = solid_capacity(m, m->host_step + nsteps)) != MFDM_OK) return rc;
  if ((rc = solid_enqueue_steps(m, nsteps)) != MFDM_OK) return rc;
  MFDM_CU(cudaStreamSynchronize(m->stream));
  int st = 0;
  MFDM_CU(cudaMemcpy(&st, m->C.status, sizeof(int), cudaMemcpyDeviceToHost));
  return status_error(st, "non-finite values reached the receiver row");
}

int mfdm_solid_time_steps(mfdm_solid* m, int nsteps, float* total_ms) {
  if (!m || !total_ms) return fail(MFDM_ERR_ARG, "null argument");
  if (nsteps < 0) return fail(MFDM_ERR_ARG, "negative step count");
  DeviceGuard g(m->device);
  int rc;
  if ((rc = solid_capacity(m, m->host_step + nsteps)) != MFDM_OK) return rc;
  cudaEvent_t e[2] = {};
  MFDM_CU(cudaEventCreate(&e[0]));
  struct Free { cudaEvent_t* e; ~Free() { for (int i = 0; i < 2; ++i) if (e[i]) cudaEventDestroy(e[i]); } } fr{e};
  MFDM_CU(cudaEventCreate(&e[1]));
  MFDM_CU(cudaEventRecord(e[0], m->stream));
  if ((rc = solid_enqueue_steps(m, nsteps)) != MFDM_OK) return rc;
  MFDM_CU(cudaEventRecord(e[1], m->stream));
  MFDM_CU(cudaEventSynchronize(e[1]));
  MFDM_CU(cudaEventElapsedTime(total_ms, e[0], e[1]));
  return MFDM_OK;
}

int mfdm_solid_get_records(mfdm_solid* m, int first, int count, float* vz) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  const int avail = (m->host_step + m->gap - 1) / m->gap;
  if (first < 0 || count < 0 || first + count > avail || first + count > m->rec_cap)
    return fail(MFDM_ERR_ARG, "record range out of bounds");
  if (count == 0 || !vz) return MFDM_OK;
  DeviceGuard g(m->device);
  MFDM_CU(cudaMemcpyAsync(vz, m->d_rec + size_t(first) * m->nx, size_t(count) * m->nx * sizeof(float),
                          cudaMemcpyDeviceToHost, m->stream));
  MFDM_CU(cudaStreamSynchronize(m->stream));
  return MFDM_OK;
}

int mfdm_solid_get_field(mfdm_solid* m, int field, float* host) {
  if (!m || !host) return fail(MFDM_ERR_ARG, "null argument");
  float* p = nullptr;
  int rc = solid_field_ptr(m, field, &p);
  if (rc != MFDM_OK) return rc;
  DeviceGuard g(m->device);
  MFDM_CU(cudaMemcpy2DAsync(host, size_t(m->nx) * sizeof(float), p, size_t(m->P) * sizeof(float),
                            size_t(m->nx) * sizeof(float), size_t(m->nz), cudaMemcpyDeviceToHost,
                            m->stream));
  MFDM_CU(cudaStreamSynchronize(m->stream));
  return MFDM_OK;
}

int mfdm_solid_get_info(const mfdm_solid* m, int* nx, int* nz, int* gap, int* step) {
  if (!m) return fail(MFDM_ERR_ARG, "null handle");
  if (nx) *nx = m->nx;
  if (nz) *nz = m->nz;
  if (gap) *gap = m->gap;
  if (step) *step = m->host_step;
  return MFDM_OK;
}

int mfdm_solid_close(mfdm_solid* m) {
  solid_destroy(m);
  return MFDM_OK;
}

}  // extern "C"

// ---- drop-in command line (src/main.cu:58-339) -------------------------------

namespace {

int write_floats(const fs::path& file, const float* data, size_t n, bool append) {
  std::ofstream f(file, std::ios::binary | (append ? std::ios::app : std::ios::trunc));
  if (!f) return fail(MFDM_ERR_IO, "cannot write " + file.string());
  f.write(reinterpret_cast<const char*>(data), std::streamsize(n * sizeof(float)));
  if (!f) return fail(MFDM_ERR_IO, "failed to write " + file.string());
  return MFDM_OK;
}

int make_dirs(const fs::path& p) {
  std::error_code ec;
  fs::create_directories(p, ec);
  if (ec) return fail(MFDM_ERR_IO, "cannot create " + p.string() + ": " + ec.message());
  return MFDM_OK;
}

// Asynchronous snapshot drain (src/main.cu:227-243, 327-339 write the files
// synchronously between steps). At a snapshot step the fields of every shot
// are copied device to device into a staging slot on the compute stream, so
// the stepping goes on at once; a copy stream moves the slot to pinned host
// memory and a worker thread writes the files <field>_%06d.bin. Two slots: the
// third snapshot waits for the first one's files. Fields: solid and fluid vx,
// vz as the reference, plus fluid p when `pressure` (documented in docs/io.md
// but not written by the reference).
class SnapshotDrain {
 public:
  ~SnapshotDrain() {
    for (auto& j : job_)
      if (j.valid()) j.wait();
    if (m_) {
      DeviceGuard g(m_->device);
      for (int s = 0; s < 2; ++s) {
        if (dev_[s]) cudaFree(dev_[s]);
        if (host_[s]) cudaFreeHost(host_[s]);
        if (staged_[s]) cudaEventDestroy(staged_[s]);
        if (copied_[s]) cudaEventDestroy(copied_[s]);
      }
      if (copy_) cudaStreamDestroy(copy_);
    }
  }

  int init(mfdm_model* m, bool pressure) {
    m_ = m;
    items_ = {{MFDM_SOLID_VZ, "solid", "vz"}, {MFDM_SOLID_VX, "solid", "vx"},
              {MFDM_FLUID_VZ, "fluid", "vz"}, {MFDM_FLUID_VX, "fluid", "vx"}};
    if (pressure) items_.push_back({MFDM_FLUID_P, "fluid", "p"});
    per_shot_ = 0;
    for (const Item& it : items_) per_shot_ += size_t(rows_of(it.field)) * m->cfg.nx;
    const size_t n = per_shot_ * size_t(m->nshots);
    DeviceGuard g(m->device);
    MFDM_CU(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
    for (int s = 0; s < 2; ++s) {
      MFDM_CU(cudaMalloc(&dev_[s], n * sizeof(float)));
      MFDM_CU(cudaMallocHost(&host_[s], n * sizeof(float)));
      MFDM_CU(cudaEventCreateWithFlags(&staged_[s], cudaEventDisableTiming));
      MFDM_CU(cudaEventCreateWithFlags(&copied_[s], cudaEventDisableTiming));
    }
    return MFDM_OK;
  }

  // Snapshot of step `it` of every shot of the handle; shot b's files go under dirs[b].
  int push(const std::vector<fs::path>& dirs, int it) {
    const int s = next_;
    next_ ^= 1;
    int rc = wait(s);
    if (rc != MFDM_OK) return rc;
    DeviceGuard g(m_->device);
    const int nx = m_->cfg.nx;
    size_t off = 0;
    for (int b = 0; b < m_->nshots; ++b)
      for (const Item& item : items_) {
        float* p = nullptr;
        int rows = 0;
        if ((rc = field_ptr(m_, item.field, &p, &rows, b)) != MFDM_OK) return rc;
        MFDM_CU(cudaMemcpy2DAsync(dev_[s] + off, size_t(nx) * sizeof(float), p,
                                  size_t(m_->P) * sizeof(float), size_t(nx) * sizeof(float),
                                  size_t(rows), cudaMemcpyDeviceToDevice, m_->stream));
        off += size_t(rows) * nx;
      }
    MFDM_CU(cudaEventRecord(staged_[s], m_->stream));
    MFDM_CU(cudaStreamWaitEvent(copy_, staged_[s], 0));
    MFDM_CU(cudaMemcpyAsync(host_[s], dev_[s], off * sizeof(float), cudaMemcpyDeviceToHost, copy_));
    MFDM_CU(cudaEventRecord(copied_[s], copy_));
    const float* host = host_[s];
    cudaEvent_t done = copied_[s];
    const std::vector<Item> items = items_;
    const int nshots = m_->nshots, device = m_->device;
    std::vector<int> rows(items.size());
    for (size_t q = 0; q < items.size(); ++q) rows[q] = rows_of(items[q].field);
    job_[s] = std::async(std::launch::async, [=]() -> Result {
      cudaSetDevice(device);
      const cudaError_t e = cudaEventSynchronize(done);
      if (e != cudaSuccess)
        return {MFDM_ERR_CUDA, std::string("snapshot copy: ") + cudaGetErrorString(e)};
      size_t o = 0;
      for (int b = 0; b < nshots; ++b)
        for (size_t q = 0; q < items.size(); ++q) {
          const fs::path dir = dirs[size_t(b)] / "snapshot" / items[q].medium / items[q].comp;
          std::error_code ec;
          fs::create_directories(dir, ec);
          if (ec) return {MFDM_ERR_IO, "cannot create " + dir.string() + ": " + ec.message()};
          std::ostringstream name;
          name << items[q].comp << "_" << std::setw(6) << std::setfill('0') << it << ".bin";
          const size_t n = size_t(rows[q]) * nx;
          std::ofstream f(dir / name.str(), std::ios::binary | std::ios::trunc);
          if (!f) return {MFDM_ERR_IO, "cannot write " + (dir / name.str()).string()};
          f.write(reinterpret_cast<const char*>(host + o), std::streamsize(n * sizeof(float)));
          if (!f) return {MFDM_ERR_IO, "failed to write " + (dir / name.str()).string()};
          o += n;
        }
      return {MFDM_OK, ""};
    });
    return MFDM_OK;
  }

  // Waits for every pending write; the first failure.
  int finish() {
    int rc = MFDM_OK;
    for (int s = 0; s < 2; ++s) {
      const int r = wait(s);
      if (rc == MFDM_OK) rc = r;
    }
    return rc;
  }

 private:
  struct Item { int field; const char* medium; const char* comp; };
  struct Result { int code; std::string msg; };
  int rows_of(int field) const { return field < 3 ? m_->cfg.nzf : m_->cfg.nzs; }
  int wait(int s) {
    if (!job_[s].valid()) return MFDM_OK;
    const Result r = job_[s].get();
    return r.code == MFDM_OK ? MFDM_OK : fail(r.code, r.msg);
  }
  mfdm_model* m_ = nullptr;
  cudaStream_t copy_ = nullptr;
  std::vector<Item> items_;
  size_t per_shot_ = 0;
  float* dev_[2] = {nullptr, nullptr};
  float* host_[2] = {nullptr, nullptr};
  cudaEvent_t staged_[2] = {nullptr, nullptr}, copied_[2] = {nullptr, nullptr};
  std::future<Result> job_[2];
  int next_ = 0;
};

bool env_on(const char* name) {
  const char* v = std::getenv(name);
  return v && *v && std::strcmp(v, "0") != 0;
}

// Steps the handle's current shot(s) through nt steps, draining a snapshot of
// every shot at each it % snapshot == 0, then writes each shot's records.
int run_shots_cli(mfdm_model* m, const std::vector<fs::path>& dirs) {
  const HostModel& h = m->cfg;
  const int nx = h.nx;
  int rc;
  for (const fs::path& d : dirs) {
    if ((rc = make_dirs(d / "snapshot")) != MFDM_OK) return rc;
    if ((rc = make_dirs(d / "record")) != MFDM_OK) return rc;
  }
  SnapshotDrain drain;
  if ((rc = drain.init(m, env_on("MFDM_SNAPSHOT_PRESSURE"))) != MFDM_OK) return rc;
  int it = 0;
  while (it < h.nt) {
    // run through the next snapshot step (it % snapshot == 0), inclusive
    const int next_snap = ((it + h.snapshot - 1) / h.snapshot) * h.snapshot;
    const int last = std::min(h.nt - 1, next_snap);
    if ((rc = mfdm_step(m, last - it + 1)) != MFDM_OK) return rc;
    it = last + 1;
    if (last % h.snapshot == 0) {
      std::printf("finished %0.2f%%\r", 100.0 * last / h.nt);
      std::fflush(stdout);
      if ((rc = drain.push(dirs, last)) != MFDM_OK) return rc;
    }
  }
  const int ns = (h.nt + m->gap - 1) / m->gap;
  std::vector<float> a(size_t(ns) * nx), b(size_t(ns) * nx), c(size_t(ns) * nx);
  for (size_t k = 0; k < dirs.size(); ++k) {
    if (ns > 0 && (rc = get_records(m, int(k), 0, ns, a.data(), b.data(), c.data())) != MFDM_OK)
      return rc;
    const fs::path rd = dirs[k] / "record";
    if ((rc = write_floats(rd / "solid_vx.bin", a.data(), a.size(), false)) != MFDM_OK) return rc;
    if ((rc = write_floats(rd / "solid_vz.bin", b.data(), b.size(), false)) != MFDM_OK) return rc;
    if ((rc = write_floats(rd / "fluid_p.bin", c.data(), c.size(), false)) != MFDM_OK) return rc;
  }
  return drain.finish();
}

int clear_out_root(const fs::path& out_root) {
  const std::string s = out_root.string();
  if (s.empty() || s == "/" || s == "." || s == "..")
    return fail(MFDM_ERR_ARG, "Invalid output dir: " + s);
  std::error_code ec;
  fs::remove_all(out_root, ec);
  if (ec) return fail(MFDM_ERR_IO, "cannot clear " + s + ": " + ec.message());
  int rc;
  if ((rc = make_dirs(out_root)) != MFDM_OK) return rc;
  std::printf("[output] cleared %s\n", s.c_str());
  return MFDM_OK;
}

void print_pml(const HostModel& h) {
  std::printf("[PML] beta0 = %.3f, p_beta = %.2f, p_alpha = %.2f, alpha0 = %.1f 1/s, d0 = %.1f 1/s\n",
              h.beta0, 2.0, 1.0, 2.0 * M_PI * h.fpeak,
              -(h.npow + 1) * double(h.vp_max) * std::log(double(h.rc)) / (2.0 * h.thickness));
}

// Solid-only runs (calc_type 0): records hold solid vz on row 3 only and the
// snapshots solid vx, vz (src/main.cu:252-339); shots carry the wavefield over
// like the fluid-solid path.
int run_cli_solid(const char* json_path, const fs::path& out_root, int device) {
  mfdm_solid* m = nullptr;
  int rc = mfdm_solid_open_json(json_path, device, &m);
  if (rc != MFDM_OK) return rc;
  struct Closer { mfdm_solid* m; ~Closer() { mfdm_solid_close(m); } } closer{m};
  print_pml(m->pml);
  if ((rc = clear_out_root(out_root)) != MFDM_OK) return rc;
  const int nx = m->nx, nz = m->nz, nt = m->nt, snap = m->snapshot;
  std::vector<float> buf(size_t(nx) * nz);
  for (int isrc = 0; isrc < std::max(1, int(m->srcx.size())); ++isrc) {
    if (m->srcx.empty()) break;
    if ((rc = mfdm_solid_set_shot(m, isrc, 0)) != MFDM_OK) return rc;
    const fs::path dir = out_root / std::to_string(isrc);
    if ((rc = make_dirs(dir / "snapshot")) != MFDM_OK) return rc;
    if ((rc = make_dirs(dir / "record")) != MFDM_OK) return rc;
    int it = 0;
    while (it < nt) {
      const int next_snap = ((it + snap - 1) / snap) * snap;
      const int last = std::min(nt - 1, next_snap);
      if ((rc = mfdm_solid_step(m, last - it + 1)) != MFDM_OK) return rc;
      it = last + 1;
      if (last % snap == 0) {
        std::printf("finished %0.2f%%\r", 100.0 * last / nt);
        std::fflush(stdout);
        const struct { int field; const char* comp; } items[] = {{MFDM_SOLID_VZ, "vz"}, {MFDM_SOLID_VX, "vx"}};
        for (const auto& item : items) {
          if ((rc = mfdm_solid_get_field(m, item.field, buf.data())) != MFDM_OK) return rc;
          const fs::path d = dir / "snapshot" / "solid" / item.comp;
          if ((rc = make_dirs(d)) != MFDM_OK) return rc;
          std::ostringstream name;
          name << item.comp << "_" << std::setw(6) << std::setfill('0') << last << ".bin";
          if ((rc = write_floats(d / name.str(), buf.data(), buf.size(), false)) != MFDM_OK) return rc;
        }
      }
    }
    const int ns = (nt + m->gap - 1) / m->gap;
    std::vector<float> rec(size_t(ns) * nx);
    if (ns > 0 && (rc = mfdm_solid_get_records(m, 0, ns, rec.data())) != MFDM_OK) return rc;
    if ((rc = write_floats(dir / "record" / "solid_vz.bin", rec.data(), rec.size(), false)) != MFDM_OK)
      return rc;
  }
  return MFDM_OK;
}

int run_cli(const char* json_path, const char* out_root_c, int device) {
  const fs::path out_root = out_root_c;
  const std::string s = out_root.string();
  if (s.empty() || s == "/" || s == "." || s == "..")
    return fail(MFDM_ERR_ARG, "Invalid output dir: " + s);
  int calc_type = 1;
  int rc0 = json_calc_type(json_path, &calc_type);
  if (rc0 != MFDM_OK) return rc0;
  if (calc_type == 0) return run_cli_solid(json_path, out_root, device);
  mfdm_model* m = nullptr;
  int rc = mfdm_open_json(json_path, device, &m);
  if (rc != MFDM_OK) return rc;
  struct Closer { mfdm_model* m; ~Closer() { mfdm_close(m); } } closer{m};
  print_pml(m->cfg);
  if ((rc = clear_out_root(out_root)) != MFDM_OK) return rc;
  const int nsrc = int(m->cfg.srcx.size());
  for (int isrc = 0; isrc < nsrc; ++isrc) {
    // The reference keeps the wavefield across shots (src/main.cu:94-136).
    if ((rc = mfdm_set_shot(m, isrc, 0)) != MFDM_OK) return rc;
    if ((rc = run_shots_cli(m, {out_root / std::to_string(isrc)})) != MFDM_OK) return rc;
  }
  return MFDM_OK;
}

// Every source of the JSON as one batch: each shot from rest, all shots in
// one launch per RK stage, a <shot>/ tree per shot.
int run_cli_batch(const char* json_path, const char* out_root_c, int device) {
  const fs::path out_root = out_root_c;
  HostModel h;
  int rc = load_json(json_path, h);
  if (rc != MFDM_OK) return rc;
  if (h.srcx.empty()) return fail(MFDM_ERR_CONFIG, "the JSON lists no source");
  std::vector<ShotCfg> shots(h.srcx.size());
  for (size_t b = 0; b < shots.size(); ++b) {
    shots[b].x = h.srcx[b];
    shots[b].z = h.srcz[b];
    shots[b].fpeak = h.fpeak;
    shots[b].beta0 = h.beta0;
  }
  print_pml(h);
  mfdm_model* m = nullptr;
  if ((rc = open_common(std::move(h), device, &m, &shots)) != MFDM_OK) return rc;
  struct Closer { mfdm_model* m; ~Closer() { mfdm_close(m); } } closer{m};
  if ((rc = clear_out_root(out_root)) != MFDM_OK) return rc;
  std::vector<fs::path> dirs;
  for (size_t b = 0; b < shots.size(); ++b) dirs.push_back(out_root / std::to_string(b));
  return run_shots_cli(m, dirs);
}

}  // namespace

extern "C" int mfdm_run_cli(const char* json_path, const char* out_root, int device) {
  if (!json_path || !out_root) return fail(MFDM_ERR_ARG, "null argument");
  try {
    return run_cli(json_path, out_root, device);
  } catch (const std::exception& e) {
    return fail(MFDM_ERR_IO, e.what());
  }
}

extern "C" int mfdm_run_cli_batch(const char* json_path, const char* out_root, int device) {
  if (!json_path || !out_root) return fail(MFDM_ERR_ARG, "null argument");
  try {
    return run_cli_batch(json_path, out_root, device);
  } catch (const std::exception& e) {
    return fail(MFDM_ERR_IO, e.what());
  }
}
