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
//   [0, nbi)          interface strip: one thread per column, fluid row nz_f-1
//                     and solid row 0 together, so the normal/tangential
//                     coupling happens in registers.
//   [nbi, nbi+nbf)    fluid segments: a 64-column strip of up to `seg` fluid rows
//                     (rows 3..nz_f-2; seg is 24 unless tuned per model)
//   [nbi+nbf, ...)    solid segments: the same over solid rows 1..nz_s-4
// With several shots the launch is one-dimensional with the shot fastest
// (blockIdx.x = block * nshots + shot), so the shots of one segment run side
// by side and all but the first read the segment's coefficients from L2.
//
// A segment block is a producer/consumer pipeline. Lane 0 of warp 8 streams the
// segment down in chunks of kR rows with 3-D TMA boxes (cp.async.bulk.tensor)
// completing on the chunk slot's mbarrier: all stencil fields of the stage
// input with a 4-column halo into a row-contiguous ring (kNS chunk
// slots), and the point-wise inputs (coefficients, U^n, accumulator) into the
// slot's point-wise buffer.
// Warps 0-7 compute one cell each per chunk purely from shared memory and
// store the stage output and accumulator straight to HBM, coalesced along x.
// Each field row thus crosses HBM once per stage; only the 3-row halo above
// and below a segment and the 4-column halo of a strip are read twice.
#include <type_traits>

#include "mfdm_async.cuh"
#include "mfdm_device.cuh"
#include "mfdm_kernels.h"

// This file is compiled twice: as it is (the stage kernels in namespace v2,
// two blocks per SM, 5 stencil and 3 point-wise ring slots, 96 registers) and
// by mfdm_kernels_b3.cu (namespace v3, three blocks per SM, 4 + 2 slots, 72
// registers). The shared kernels and the dispatching launchers are built once.
#ifndef MFDM_VNS
#define MFDM_VNS v2
#endif

namespace mfdm {
namespace MFDM_VNS {

constexpr int kTX = kStageTX;            // computed columns per strip
constexpr int kSW = kStageSW;            // staged row width (4-column halo each side)
constexpr int kR = kStageR;              // rows per chunk
#ifndef MFDM_STENCIL_SLOTS
#define MFDM_STENCIL_SLOTS 5
#endif
#ifndef MFDM_PW_SLOTS
#define MFDM_PW_SLOTS 3
#endif
#ifndef MFDM_MIN_BLOCKS
#define MFDM_MIN_BLOCKS 2  // stage blocks resident per SM (registers: 96 at 2)
#endif
constexpr int kNS = MFDM_STENCIL_SLOTS;   // stencil chunk slots
constexpr int kNP = MFDM_PW_SLOTS;        // point-wise chunk slots
constexpr int kRing = kR * kNS;          // ring rows
constexpr int kConsumers = 256;          // warps 0-7
constexpr int kThreads = kConsumers + 32;  // + producer warp
constexpr int kBarBytes = 256;           // full/empty barriers of both rings


static_assert(kTX * kR == kConsumers, "one cell per consumer thread per chunk");
// The stencil ring is row-contiguous ([ring row][field][col]) with kR extra rows
// on each side: the chunk in the last slot is also copied above the first slot
// and the chunk in the first slot below the last one, so the rows dz = -3..3
// around any ring row are contiguous and no read wraps around.
constexpr int kRingRows = kRing + 2 * kR;
static_assert(kNS >= 3 && kNP >= 1, "ring depths");
static_assert(2 * (kNS + kNP) * 8 <= kBarBytes, "barrier region too small");

// Point-wise inputs staged per chunk, by stage kind: coefficients, then U^n
// (middle stages), then the accumulator (middle and last stages).
template <int NST, int NCOEF, int KIND>
struct PW {
  static constexpr int n = NCOEF + (KIND == kStageMid ? 2 * NST : (KIND == kStageLast ? NST : 0));
};

// Shared memory of one segment block: barriers, the stencil ring of kRingRows
// rows [NST][kSW], kNP point-wise slots of [NPW][kR][kTX] (all 128-byte
// multiples), plus 128 bytes to align the dynamic base.
template <int NST, int NPW>
__host__ __device__ constexpr size_t segment_smem() {
  return size_t(128) + kBarBytes + size_t(kRingRows) * NST * kSW * 4 +
         size_t(kNP) * NPW * kR * kTX * 4;
}

// Reads the stage input from the stencil ring: the cell's ring row rr and the
// rows dz = -3..3 around it are contiguous, so every read is the cell's base
// plus a compile-time offset.
template <int NST>
struct RingAcc {
  const float* base;  // ring row (rr) of the cell, its column (with the halo)
  __device__ __forceinline__ void init(const float* ring, int rr, int c) {
    base = ring + (kR + rr) * (NST * kSW) + c;
  }
  __device__ __forceinline__ float at(int f, int dz, int dx) const {
    return base[dz * (NST * kSW) + f * kSW + dx];
  }
};
struct FluidRing : RingAcc<3> {
  __device__ __forceinline__ float fvx(int dz, int dx) const { return at(0, dz, dx); }
  __device__ __forceinline__ float fvz(int dz, int dx) const { return at(1, dz, dx); }
  __device__ __forceinline__ float fp(int dz, int dx) const { return at(2, dz, dx); }
};
struct SolidRing : RingAcc<5> {
  __device__ __forceinline__ float svx(int dz, int dx) const { return at(0, dz, dx); }
  __device__ __forceinline__ float svz(int dz, int dx) const { return at(1, dz, dx); }
  __device__ __forceinline__ float ssx(int dz, int dx) const { return at(2, dz, dx); }
  __device__ __forceinline__ float ssz(int dz, int dx) const { return at(3, dz, dx); }
  __device__ __forceinline__ float ssxz(int dz, int dx) const { return at(4, dz, dx); }
};
// Geometry of one segment block.
struct Segment {
  int x0;     // first computed column of the strip
  int z0;     // first computed row
  int z1;     // one past the last computed row
  int rows;   // rows of the arrays (fluid nz_f or solid nz_s)
  int nch;    // computed chunks
};

// The mbarriers of a segment block: the stencil ring's full/empty pair per
// slot and the point-wise ring's.
struct Bars {
  uint64_t *full, *empty, *pfull, *pempty;
};

// Producer (one lane of warp 8). Stencil chunk k (k = -1 .. nch; the two ends
// carry only the halo rows) goes to ring slot (k + 1) % kNS once the slot's
// previous chunk is released: one 3-D TMA box with all stencil fields of kR
// rows and the column halo (chunks of the first and last slot a second time,
// past the ring's other end). The point-wise inputs of chunk j (j = 0 .. nch-1:
// coefficients, U^n, accumulator, up to three boxes) go to point-wise slot
// j % kNP once chunk j - kNP is computed, and are issued right after stencil
// chunk j + D, D = kNS - 1 - kNP: the two waits then become due together, so
// neither ring holds up the other.
// Tiled TMA always delivers whole boxes (zero-filled outside the arrays), so
// every byte count announced on a barrier is a compile-time constant.
template <int NST, int NCOEF, int KIND>
__device__ __forceinline__ void produce(const Segment& sg, const CUtensorMap* in_map,
                                        const CUtensorMap* coef_map, const CUtensorMap* un_map,
                                        const CUtensorMap* acc_map, float* ring, float* slots,
                                        const Bars& B, int* status, int shot) {
  if ((threadIdx.x & 31) != 0) return;
  constexpr int NPW = PW<NST, NCOEF, KIND>::n;
  constexpr unsigned kStBytes = NST * kR * kSW * 4, kPwBytes = NPW * kR * kTX * 4;
  constexpr int kRowF = NST * kSW;  // floats per ring row
  constexpr int kF = kR * kTX;      // floats per point-wise field in a slot
  constexpr int D = kNS - 1 - kNP;
  auto issue_pw = [&](int j) -> bool {
    const int ps = j % kNP;
    if (j >= kNP && !mbar_wait(&B.pempty[ps], ((j / kNP) - 1) & 1)) return false;
    const int q0 = sg.z0 + j * kR;
    float* d = slots + ps * NPW * kF;
    mbar_arrive_expect_tx(&B.pfull[ps], kPwBytes);
    tma_load_3d(d, coef_map, sg.x0, q0, 0, &B.pfull[ps]);
    if (KIND == kStageMid) {
      tma_load_4d(d + NCOEF * kF, un_map, sg.x0, q0, 0, shot, &B.pfull[ps]);
      tma_load_4d(d + (NCOEF + NST) * kF, acc_map, sg.x0, q0, 0, shot, &B.pfull[ps]);
    } else if (KIND == kStageLast) {
      tma_load_4d(d + NCOEF * kF, acc_map, sg.x0, q0, 0, shot, &B.pfull[ps]);
    }
    return true;
  };
  for (int k = -1; k <= sg.nch; ++k) {
    const int u = k + 1, slot = u % kNS;
    if (u >= kNS && !mbar_wait(&B.empty[slot], ((u / kNS) - 1) & 1)) {
      atomicOr(status, 2);
      return;
    }
    const int r0 = sg.z0 + k * kR;
    const bool dup = slot == 0 || slot == kNS - 1;  // also copied past the ring's other end
    mbar_arrive_expect_tx(&B.full[slot], kStBytes * (dup ? 2u : 1u));
    tma_load_4d(ring + (kR + slot * kR) * kRowF, in_map, sg.x0 - 4, 0, r0, shot, &B.full[slot]);
    if (dup)
      tma_load_4d(ring + (slot == 0 ? kR + kRing : 0) * kRowF, in_map, sg.x0 - 4, 0, r0, shot,
                  &B.full[slot]);
    const int j = k - D;  // point-wise chunk due with stencil chunk k
    if (j >= 0 && j < sg.nch && !issue_pw(j)) {
      atomicOr(status, 2);
      return;
    }
  }
  for (int j = (sg.nch + 1 - D > 0 ? sg.nch + 1 - D : 0); j < sg.nch; ++j) {
    if (!issue_pw(j)) {
      atomicOr(status, 2);
      return;
    }
  }
}

// Consumer side of the pipeline: per chunk c waits for stencil chunk c+1 (the
// halo below chunk c) and point-wise chunk c, hands each thread its cell, then
// releases stencil chunk c-1 and point-wise chunk c.
template <class Body>
__device__ __forceinline__ void consume(const Segment& sg, const Bars& B, int* status,
                                        const Body& body) {
  const int lane = threadIdx.x & 31;
  // stencil chunks -1 and 0 (slots 0 and 1, first use)
  if (!mbar_wait(&B.full[0], 0) || !mbar_wait(&B.full[1], 0)) {
    if (lane == 0) atomicOr(status, 2);
    return;
  }
  for (int c = 0; c < sg.nch; ++c) {
    const int un = c + 2;  // stencil use of chunk c+1
    if (!mbar_wait(&B.full[un % kNS], (un / kNS) & 1) ||
        !mbar_wait(&B.pfull[c % kNP], (c / kNP) & 1)) {
      if (lane == 0) atomicOr(status, 2);
      return;
    }
    body(c, c % kNP);
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(&B.empty[c % kNS]);  // stencil chunk c-1 is no longer needed
      mbar_arrive(&B.pempty[c % kNP]);
    }
  }
}

// Carves the barriers and the slots out of the dynamic shared memory (base
// rounded up to 128 bytes) and initialises the barriers.
template <int NST>
__device__ __forceinline__ void segment_setup(char* smem_raw, Bars& B, float*& ring, float*& slots) {
  char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  B.full = reinterpret_cast<uint64_t*>(smem);
  B.empty = B.full + kNS;
  B.pfull = B.empty + kNS;
  B.pempty = B.pfull + kNP;
  ring = reinterpret_cast<float*>(smem + kBarBytes);
  slots = ring + kRingRows * NST * kSW;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kNS; ++i) {
      mbar_init(&B.full[i], 1);
      mbar_init(&B.empty[i], kConsumers / 32);
    }
    for (int i = 0; i < kNP; ++i) {
      mbar_init(&B.pfull[i], 1);
      mbar_init(&B.pempty[i], kConsumers / 32);
    }
    mbar_fence_init();
  }
  __syncthreads();
}

template <int DIR, int KIND, bool CPML>
__device__ __forceinline__ void fluid_segment(const Coef& C, const Fields& in, const Fields& out,
                                              const Fields& un, const Fields& acc,
                                              const StageMaps& maps, int s, float cc, float w,
                                              int blk, int ntx, int seg, int shot, char* smem) {
  constexpr int NST = 3, NCOEF = 6, NPW = PW<NST, NCOEF, KIND>::n;
  const int P = C.P, nx = C.nx;
  Segment sg;
  sg.x0 = (blk % ntx) * kTX;
  sg.z0 = 3 + (blk / ntx) * seg;
  sg.z1 = min(sg.z0 + seg, C.nzf - 1);
  sg.rows = C.nzf;
  sg.nch = (sg.z1 - sg.z0 + kR - 1) / kR;
  Bars B;
  float *ring, *slots;
  segment_setup<NST>(smem, B, ring, slots);
  const int it = __ldg(C.step);
  if (threadIdx.x >= kConsumers) {
    produce<NST, NCOEF, KIND>(sg, &maps.fin, &maps.fcoef, &maps.fun, &maps.facc, ring, slots, B,
                              C.status, shot);
    return;
  }
  const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
  const int ix = sg.x0 + tx;
  const bool colok = ix >= 3 && ix <= nx - 4;
  const bool side = colok && min(ix - 3, nx - 4 - ix) < C.npd;
  const int scol = side ? xstrip_col(ix, nx, C.npd) : 0;
  // Segments with no side-strip cell, no edge column, no source cell and no
  // conservative or one-sided row (rows 6 .. nz_f-4 only) take a body without
  // those branches.
  const bool general = sg.x0 < 3 + C.npd || sg.x0 + kTX > nx - 3 - C.npd ||
                       sg.z0 < 6 || sg.z1 - 1 > C.nzf - 4 || (CPML && sg.z0 <= C.npd + 2) ||
                       (C.srcx >= 0 && C.srcx >= sg.x0 - 2 && C.srcx < sg.x0 + kTX + 2 &&
                        C.srcz >= sg.z0 - 2 && C.srcz < sg.z1 + 2);
  auto cell = [&](auto gen_tag, int c, int slot) {
    constexpr bool GEN = decltype(gen_tag)::value;
    const int iz = sg.z0 + c * kR + ty;
    if ((GEN && !colok) || iz >= sg.z1) return;
    const bool sd = GEN && side;  // a side-strip cell
    FluidRing A;
    A.init(ring, ((c + 1) % kNS) * kR + ty, tx + 4);
    constexpr int F = kR * kTX;
    const float* pw = slots + (size_t)slot * NPW * F + ty * kTX + tx;  // field p at pw[p * F]
    const FluidCoefs cf{pw[0], pw[F], pw[2 * F], pw[3 * F], pw[4 * F], pw[5 * F]};
    float ade[4] = {0.f, 0.f, 0.f, 0.f}, zade[4] = {0.f, 0.f, 0.f, 0.f};
    const size_t si = (size_t)iz * C.Ps + scol;
    if (sd) {
#pragma unroll
      for (int q = 0; q < 4; ++q) ade[q] = __ldg(in.fx[q] + si);
    }
    // four-side CPML: the top zeta band, rows 3..npd+2, strip row iz - 3
    const bool tp = GEN && CPML && iz <= C.npd + 2;
    const size_t zi = (size_t)(iz - 3) * P + ix;
    if (tp) {
#pragma unroll
      for (int q = 0; q < 4; ++q) zade[q] = __ldg(in.fz[q] + zi);
    }
    // rows 6 .. nz_f-4 take the specialised interior body (no conservative rows)
    FluidK k = (!GEN || (iz >= 6 && iz <= C.nzf - 4))
                   ? fluid_rhs<DIR, true, CPML>(C, A, iz, ix, sd, ade, cf, tp, zade)
                   : fluid_rhs<DIR, false, CPML>(C, A, iz, ix, sd, ade, cf, tp, zade);
    if (GEN) k.p += source_term(C, iz, ix, it, s);
    const size_t i = (size_t)iz * P + ix;
    const float kv[3] = {k.vx, k.vz, k.p};
    float* const outs[3] = {out.fvx, out.fvz, out.fp};
    float* const accs[3] = {acc.fvx, acc.fvz, acc.fp};
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      if (KIND == kStageFirst) {
        const float u0 = A.at(f, 0, 0);
        outs[f][i] = fmaf(cc, kv[f], u0);
        accs[f][i] = fmaf(w, kv[f], u0);
      } else if (KIND == kStageMid) {
        outs[f][i] = fmaf(cc, kv[f], pw[(NCOEF + f) * F]);
        accs[f][i] = fmaf(w, kv[f], pw[(NCOEF + NST + f) * F]);
      } else {
        outs[f][i] = fmaf(cc, kv[f], pw[(NCOEF + f) * F]);
      }
    }
    if (sd) {
      rk_update<KIND>(k.V0, ade[0], un.fx[0], out.fx[0], acc.fx[0], si, cc, w);
      rk_update<KIND>(k.V1, ade[1], un.fx[1], out.fx[1], acc.fx[1], si, cc, w);
      if (k.has_E) {
        rk_update<KIND>(k.E0, ade[2], un.fx[2], out.fx[2], acc.fx[2], si, cc, w);
        rk_update<KIND>(k.E1, ade[3], un.fx[3], out.fx[3], acc.fx[3], si, cc, w);
      }
    }
    if (tp) {
      rk_update<KIND>(k.ZV0, zade[0], un.fz[0], out.fz[0], acc.fz[0], zi, cc, w);
      rk_update<KIND>(k.ZV1, zade[1], un.fz[1], out.fz[1], acc.fz[1], zi, cc, w);
      rk_update<KIND>(k.ZE0, zade[2], un.fz[2], out.fz[2], acc.fz[2], zi, cc, w);
      rk_update<KIND>(k.ZE1, zade[3], un.fz[3], out.fz[3], acc.fz[3], zi, cc, w);
    }
  };
  if (general)
    consume(sg, B, C.status, [&](int c, int slot) { cell(std::true_type{}, c, slot); });
  else
    consume(sg, B, C.status, [&](int c, int slot) { cell(std::false_type{}, c, slot); });
}

template <int DIR, int KIND, bool CPML>
__device__ __forceinline__ void solid_segment(const Coef& C, const Fields& in, const Fields& out,
                                              const Fields& un, const Fields& acc,
                                              const StageMaps& maps, float cc, float w, int blk,
                                              int ntx, int seg, int shot, char* smem) {
  constexpr int NST = 5, NCOEF = 9, NPW = PW<NST, NCOEF, KIND>::n;
  const int P = C.P, nx = C.nx, npd = C.npd, nzs = C.nzs;
  Segment sg;
  sg.x0 = (blk % ntx) * kTX;
  sg.z0 = 1 + (blk / ntx) * seg;
  sg.z1 = min(sg.z0 + seg, nzs - 3);
  sg.rows = nzs;
  sg.nch = (sg.z1 - sg.z0 + kR - 1) / kR;
  Bars B;
  float *ring, *slots;
  segment_setup<NST>(smem, B, ring, slots);
  if (threadIdx.x >= kConsumers) {
    produce<NST, NCOEF, KIND>(sg, &maps.sin, &maps.scoef, &maps.sun, &maps.sacc, ring, slots, B,
                              C.status, shot);
    return;
  }
  const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
  const int ix = sg.x0 + tx;
  const bool colok = ix >= 3 && ix <= nx - 4;
  const bool side = colok && min(ix - 3, nx - 4 - ix) < npd;
  const int scol = side ? xstrip_col(ix, nx, npd) : 0;
  const int zb0 = nzs - 3 - npd;  // first row of the bottom strip
  // Segments with no PML cell, no edge column and no flux-form row (rows >= 3
  // only) take a body without those branches.
  const bool general = sg.x0 < 3 + npd || sg.x0 + kTX > nx - 3 - npd || sg.z1 > zb0 || sg.z0 < 3;
  auto cell = [&](auto gen_tag, int c, int slot) {
    constexpr bool GEN = decltype(gen_tag)::value;
    const int iz = sg.z0 + c * kR + ty;
    if ((GEN && !colok) || iz >= sg.z1) return;
    const bool sd = GEN && side;  // a side-strip cell
    const bool bottom = GEN && iz >= zb0;
    SolidRing A;
    A.init(ring, ((c + 1) % kNS) * kR + ty, tx + 4);
    constexpr int F = kR * kTX;
    const float* pw = slots + (size_t)slot * NPW * F + ty * kTX + tx;
    const SolidCoefs cf{pw[0], pw[F], pw[2 * F], pw[3 * F], pw[4 * F],
                        pw[5 * F], pw[6 * F], pw[7 * F], pw[8 * F]};
    float xade[4] = {0.f, 0.f, 0.f, 0.f}, zade[4] = {0.f, 0.f, 0.f, 0.f};
    const size_t sxi = (size_t)iz * C.Ps + scol;
    const size_t szi = (size_t)(iz - zb0) * P + ix;
    if (sd) {
#pragma unroll
      for (int q = 0; q < 4; ++q) xade[q] = __ldg(in.sx[q] + sxi);
    }
    if (bottom) {
#pragma unroll
      for (int q = 0; q < 4; ++q) zade[q] = __ldg(in.sz[q] + szi);
    }
    SolidK k = (!GEN || iz >= 3)
                   ? solid_rhs<DIR, true, CPML>(C, A, iz, ix, sd, bottom, xade, zade, cf)
                   : solid_rhs<DIR, false, CPML>(C, A, iz, ix, sd, bottom, xade, zade, cf);
    const size_t i = (size_t)iz * P + ix;
    const float kv[5] = {k.vx, k.vz, k.sx, k.sz, k.sxz};
    float* const outs[5] = {out.svx, out.svz, out.ssx, out.ssz, out.ssxz};
    float* const accs[5] = {acc.svx, acc.svz, acc.ssx, acc.ssz, acc.ssxz};
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      if (KIND == kStageFirst) {
        const float u0 = A.at(f, 0, 0);
        outs[f][i] = fmaf(cc, kv[f], u0);
        accs[f][i] = fmaf(w, kv[f], u0);
      } else if (KIND == kStageMid) {
        outs[f][i] = fmaf(cc, kv[f], pw[(NCOEF + f) * F]);
        accs[f][i] = fmaf(w, kv[f], pw[(NCOEF + NST + f) * F]);
      } else {
        outs[f][i] = fmaf(cc, kv[f], pw[(NCOEF + f) * F]);
      }
    }
    if (sd) {
      rk_update<KIND>(k.XV0, xade[0], un.sx[0], out.sx[0], acc.sx[0], sxi, cc, w);
      rk_update<KIND>(k.XV1, xade[1], un.sx[1], out.sx[1], acc.sx[1], sxi, cc, w);
      rk_update<KIND>(k.XE0, xade[2], un.sx[2], out.sx[2], acc.sx[2], sxi, cc, w);
      rk_update<KIND>(k.XE1, xade[3], un.sx[3], out.sx[3], acc.sx[3], sxi, cc, w);
    }
    if (bottom) {
      rk_update<KIND>(k.ZV0, zade[0], un.sz[0], out.sz[0], acc.sz[0], szi, cc, w);
      rk_update<KIND>(k.ZV1, zade[1], un.sz[1], out.sz[1], acc.sz[1], szi, cc, w);
      rk_update<KIND>(k.ZE0, zade[2], un.sz[2], out.sz[2], acc.sz[2], szi, cc, w);
      rk_update<KIND>(k.ZE1, zade[3], un.sz[3], out.sz[3], acc.sz[3], szi, cc, w);
    }
  };
  if (general)
    consume(sg, B, C.status, [&](int c, int slot) { cell(std::true_type{}, c, slot); });
  else
    consume(sg, B, C.status, [&](int c, int slot) { cell(std::false_type{}, c, slot); });
}

// Interface strip: fluid row nz_f-1 and solid row 0 of one column, their RHS,
// the normal/tangential coupling (pml_fs_kernels.cuh:754-827) and the RK update.
// In the last stage the eight coupled state values go to C.ipre, the filter's input.
template <int DIR, int KIND, bool CPML>
__device__ __forceinline__ void interface_strip(const Coef& C, const Fields& in, const Fields& out,
                                                const Fields& un, const Fields& acc, float c,
                                                float w, int blk) {
  const int nx = C.nx, P = C.P, nzf = C.nzf, nzs = C.nzs, npd = C.npd;
  if (threadIdx.x >= kConsumers) return;
  const int ix = blk * kConsumers + threadIdx.x;
  if (ix < 3 || ix > nx - 4) return;
  const bool side = min(ix - 3, nx - 4 - ix) < npd;
  const int scol = side ? xstrip_col(ix, nx, npd) : 0;
  const int zb0 = nzs - 3 - npd;
  const bool bottom = 0 >= zb0;

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
  // four-side CPML on a grid whose top band reaches the interface row
  const bool ftop = CPML && nzf - 1 <= npd + 2;
  float ztop[4] = {0.f, 0.f, 0.f, 0.f};
  const size_t zti = (size_t)(nzf - 1 - 3) * P + ix;
  if (ftop) {
#pragma unroll
    for (int q = 0; q < 4; ++q) ztop[q] = __ldg(in.fz[q] + zti);
  }
  FluidK kf = fluid_rhs<DIR, false, CPML>(C, Af, nzf - 1, ix, side, fade, fluid_coefs_global(C, fi),
                                          ftop, ztop);
  SolidK ks = solid_rhs<DIR, false, CPML>(C, As, 0, ix, side, bottom, xade, zade,
                             solid_coefs_global(C, si, si + (size_t)(nzf - 1) * P));

  // ---- coupling of the stage RHS on the interface ----
  const float2 n = __ldg(C.nrm + ix);
  const float kfv[3] = {kf.vx, kf.vz, kf.p}, ksv[5] = {ks.vx, ks.vz, ks.sx, ks.sz, ks.sxz};
  float kv[8];
  couple_rhs<DIR>(n, kfv, ksv, kv);
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
  if (ftop) {
    rk_update<KIND>(kf.ZV0, ztop[0], un.fz[0], out.fz[0], acc.fz[0], zti, c, w);
    rk_update<KIND>(kf.ZV1, ztop[1], un.fz[1], out.fz[1], acc.fz[1], zti, c, w);
    rk_update<KIND>(kf.ZE0, ztop[2], un.fz[2], out.fz[2], acc.fz[2], zti, c, w);
    rk_update<KIND>(kf.ZE1, ztop[3], un.fz[3], out.fz[3], acc.fz[3], zti, c, w);
  }
}

// One RK stage: `s` indexes the Ricker table; cc and w are the stage's RK
// weights (out = base + cc k, accumulator += w k).
template <int DIR, int KIND, bool CPML>
__global__ void __launch_bounds__(kThreads, MFDM_MIN_BLOCKS)
    stage_kernel(Coef C0, Fields in0, Fields out0, Fields un0, Fields acc0,
                 const __grid_constant__ StageMaps maps, int s, float cc, float w, int ntx,
                 int nbi, int nbf, int nbs, int seg, int nshots) {
  extern __shared__ char smem[];
  // this block's shot (the fastest index): its own state, tables and buffers
  const int shot = int(blockIdx.x % unsigned(nshots));
  const int b = int(blockIdx.x / unsigned(nshots));
  const size_t so = size_t(shot) * C0.shot_stride;
  const Coef C = shot_coef(C0, shot);
  const Fields in = shot_fields(in0, so), out = shot_fields(out0, so), un = shot_fields(un0, so),
               acc = shot_fields(acc0, so);
  if (b < nbi) {  // first, so the short interface blocks overlap the segments
    interface_strip<DIR, KIND, CPML>(C, in, out, un, acc, cc, w, b);
  } else if (b < nbi + nbf) {
    fluid_segment<DIR, KIND, CPML>(C, in, out, un, acc, maps, s, cc, w, b - nbi, ntx, seg, shot,
                                   smem);
  } else {
    solid_segment<DIR, KIND, CPML>(C, in, out, un, acc, maps, cc, w, b - nbi - nbf, ntx, seg, shot,
                                   smem);
  }
}

// ---- host-side launchers of this build's stage kernels ------------------------

template <int KIND>
static size_t smem_for_kind() {
  const size_t f = segment_smem<3, PW<3, 6, KIND>::n>(), so = segment_smem<5, PW<5, 9, KIND>::n>();
  return f > so ? f : so;
}

size_t smem_bytes() { return smem_for_kind<kStageMid>(); }

static int seg_rows_of(const Coef& C) { return C.seg > 0 ? C.seg : default_seg_rows(C); }

static void grid_of(int nx, int nzf, int nzs, int seg, int* ntx, int* nbf, int* nbs, int* nbi) {
  *ntx = (nx + kTX - 1) / kTX;
  const int frows = nzf - 1 - 3;  // fluid rows 3..nz_f-2
  const int srows = nzs - 4;      // solid rows 1..nz_s-4
  *nbf = frows > 0 ? *ntx * ((frows + seg - 1) / seg) : 0;
  *nbs = srows > 0 ? *ntx * ((srows + seg - 1) / seg) : 0;
  *nbi = (nx + kConsumers - 1) / kConsumers;
}

template <int DIR, int KIND, bool CPML>
static cudaError_t launch_one(const Coef& C, const Fields& in, const Fields& out, const Fields& un,
                              const Fields& acc, const StageMaps& maps, int s, cudaStream_t st) {
  int ntx, nbf, nbs, nbi;
  const int seg = seg_rows_of(C), nshots = C.nshots > 0 ? C.nshots : 1;
  grid_of(C.nx, C.nzf, C.nzs, seg, &ntx, &nbf, &nbs, &nbi);
  const float cc = C.rk_c[s], w = (KIND == kStageLast) ? 0.f : C.rk_w[s];
  const unsigned grid = unsigned(nbi + nbf + nbs) * unsigned(nshots);
  stage_kernel<DIR, KIND, CPML><<<grid, kThreads, smem_for_kind<KIND>(), st>>>(
      C, in, out, un, acc, maps, s, cc, w, ntx, nbi, nbf, nbs, seg, nshots);
  return cudaGetLastError();
}

template <int DIR, int KIND>
static cudaError_t configure_one() {
  cudaError_t e = cudaFuncSetAttribute(stage_kernel<DIR, KIND, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem_for_kind<KIND>());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(stage_kernel<DIR, KIND, true>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_for_kind<KIND>());
}

cudaError_t configure() {
  cudaError_t e;
  if ((e = configure_one<kDirF, kStageFirst>()) != cudaSuccess) return e;
  if ((e = configure_one<kDirF, kStageMid>()) != cudaSuccess) return e;
  if ((e = configure_one<kDirF, kStageLast>()) != cudaSuccess) return e;
  if ((e = configure_one<kDirB, kStageFirst>()) != cudaSuccess) return e;
  if ((e = configure_one<kDirB, kStageMid>()) != cudaSuccess) return e;
  return configure_one<kDirB, kStageLast>();
}

template <bool CPML>
static cudaError_t launch_stage_bc(const Coef& C, const Fields& in, const Fields& out,
                                  const Fields& un, const Fields& acc, const StageMaps& maps,
                                  int stage, int dir, cudaStream_t st) {
  const int kind = stage == 0 ? kStageFirst : (stage == 3 ? kStageLast : kStageMid);
  if (dir == kDirF) {
    if (kind == kStageFirst) return launch_one<kDirF, kStageFirst, CPML>(C, in, out, un, acc, maps, stage, st);
    if (kind == kStageMid) return launch_one<kDirF, kStageMid, CPML>(C, in, out, un, acc, maps, stage, st);
    return launch_one<kDirF, kStageLast, CPML>(C, in, out, un, acc, maps, stage, st);
  }
  if (kind == kStageFirst) return launch_one<kDirB, kStageFirst, CPML>(C, in, out, un, acc, maps, stage, st);
  if (kind == kStageMid) return launch_one<kDirB, kStageMid, CPML>(C, in, out, un, acc, maps, stage, st);
  return launch_one<kDirB, kStageLast, CPML>(C, in, out, un, acc, maps, stage, st);
}

cudaError_t launch_stage_v(const Coef& C, const Fields& in, const Fields& out, const Fields& un,
                           const Fields& acc, const StageMaps& maps, int stage, int dir,
                           cudaStream_t st) {
  // the four-side CPML variant runs its own kernel instantiations
  return C.cpml ? launch_stage_bc<true>(C, in, out, un, acc, maps, stage, dir, st)
                : launch_stage_bc<false>(C, in, out, un, acc, maps, stage, dir, st);
}

// The stage kernels' constant weights live in this build's own constant bank.
cudaError_t upload_constants_v(const float* srcw25, const float* w7) {
  cudaError_t e = cudaMemcpyToSymbol(c_srcw, srcw25, 25 * sizeof(float));
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_w7, w7, 7 * sizeof(float));
}

#ifndef MFDM_VARIANT_TU
// ---- the tile build: shared-memory stencil tiles and plain loads ------------------
//
// Blocks of 256 threads own 32 columns x `tr` rows of the fluid or the solid
// (tr: the segment height rounded up to a multiple of 8, at most 48; two rows
// per thread at the default 16). A block stages the stage-input fields of its cells with their 3-row,
// 4-column halo in shared memory with independent float4 loads (zero outside
// the arrays, as the tensor maps of the ring builds fill), while every thread
// already has the point-wise operands of its first row in flight: U^n, the
// accumulator and the coefficient block's values (metric copies, 1/rho and K
// or the stiffnesses). 32 warps per SM, no producer warp, no ring barriers.
// The interface strip is the ring builds' (global loads).

constexpr int kTileX = 32;                 // columns per tile block
constexpr int kTileRowsMax = 48;           // tallest tile block
constexpr int kTileW = kTileX + 8;         // staged row: columns x0-4 .. x0+35
constexpr int kTileHMax = kTileRowsMax + 6;  // staged rows: z0-3 .. z0+tr+2
constexpr int kTileThreads = 256;
constexpr int kTileRowStep = kTileThreads / kTileX;  // rows between a thread's cells (8)
#ifndef MFDM_TILE_MIN_BLOCKS
#define MFDM_TILE_MIN_BLOCKS 4  // tile blocks resident per SM (the register cap)
#endif
static_assert(kTileThreads == kConsumers, "the interface strip's blocks");

// Stage input staged as [row][field][column] (like the ring, so the same
// compile-time offsets reach every neighbour).
template <int NST>
struct TileAcc {
  const float* base;
  __device__ __forceinline__ void init(const float* tile, int lz, int c) {
    base = tile + lz * (NST * kTileW) + c;
  }
  __device__ __forceinline__ float at(int f, int dz, int dx) const {
    return base[dz * (NST * kTileW) + f * kTileW + dx];
  }
};
struct FluidTile : TileAcc<3> {
  __device__ __forceinline__ float fvx(int dz, int dx) const { return at(0, dz, dx); }
  __device__ __forceinline__ float fvz(int dz, int dx) const { return at(1, dz, dx); }
  __device__ __forceinline__ float fp(int dz, int dx) const { return at(2, dz, dx); }
};
struct SolidTile : TileAcc<5> {
  __device__ __forceinline__ float svx(int dz, int dx) const { return at(0, dz, dx); }
  __device__ __forceinline__ float svz(int dz, int dx) const { return at(1, dz, dx); }
  __device__ __forceinline__ float ssx(int dz, int dx) const { return at(2, dz, dx); }
  __device__ __forceinline__ float ssz(int dz, int dx) const { return at(3, dz, dx); }
  __device__ __forceinline__ float ssxz(int dz, int dx) const { return at(4, dz, dx); }
};

// Point-wise operands of one cell, loaded before any store of its row (the
// output and accumulator pointers may alias the inputs as far as the compiler
// knows, which would otherwise order each field's loads after the previous
// field's stores).
template <int NST, int NCOEF>
struct TilePt { float u[NST], a[NST], k[NCOEF]; };

template <int NST, int NCOEF, int KIND>
__device__ __forceinline__ void tile_load_pt(TilePt<NST, NCOEF>& p, const float* const* un,
                                             const float* const* acc, const float* coef,
                                             size_t nblk, size_t i) {
#pragma unroll
  for (int f = 0; f < NST; ++f) {
    if (KIND == kStageMid) p.u[f] = __ldg(un[f] + i);
    if (KIND != kStageFirst) p.a[f] = acc[f][i];
  }
#pragma unroll
  for (int q = 0; q < NCOEF; ++q) p.k[q] = __ldg(coef + q * nblk + i);
}

// Stage rows z0-3 .. z0+tr+2 of the NST fields (rows of `rows`, pitch P),
// columns x0-4 .. x0+35; zero where a ring build's tensor map reads zero.
template <int NST>
__device__ __forceinline__ void tile_stage(float* tile, const float* const* f, int x0, int z0,
                                           int tr, int rows, int P) {
  constexpr int kV = kTileW / 4, kPer = NST * kV;
  for (int e = threadIdx.x; e < (tr + 6) * kPer; e += kTileThreads) {
    const int rr = e / kPer, rem = e - rr * kPer, q = rem / kV, vc = (rem - q * kV) * 4;
    const int r = z0 - 3 + rr, col = x0 - 4 + vc;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (r >= 0 && r < rows && col >= 0 && col < P)
      v = __ldg(reinterpret_cast<const float4*>(f[q] + (size_t)r * P + col));
    *reinterpret_cast<float4*>(tile + (rr * NST + q) * kTileW + vc) = v;
  }
}

template <int DIR, int KIND, bool CPML>
__device__ __forceinline__ void fluid_tile(const Coef& C, const Fields& in, const Fields& out,
                                           const Fields& un, const Fields& acc, int s, float cc,
                                           float w, int blk, int ntx, int tr, float* tile) {
  constexpr int NST = 3, NCOEF = 6;
  const int P = C.P, nx = C.nx, nzf = C.nzf, npd = C.npd;
  const size_t nf = (size_t)nzf * P;
  const int x0 = (blk % ntx) * kTileX, z0 = 3 + (blk / ntx) * tr;
  const int z1 = min(z0 + tr, nzf - 1);
  const int tx = threadIdx.x % kTileX, ty = threadIdx.x / kTileX;
  const int ix = x0 + tx;
  const bool colok = ix >= 3 && ix <= nx - 4;
  const float* const uns[3] = {un.fvx, un.fvz, un.fp};
  const float* const accs_c[3] = {acc.fvx, acc.fvz, acc.fp};
  const float* coef = C.rhof - 4 * nf;  // the fluid coefficient block [6][nz_f][P]
  TilePt<NST, NCOEF> p;
  if (colok && z0 + ty < z1)
    tile_load_pt<NST, NCOEF, KIND>(p, uns, accs_c, coef, nf, (size_t)(z0 + ty) * P + ix);
  {
    const float* const f[3] = {in.fvx, in.fvz, in.fp};
    tile_stage<NST>(tile, f, x0, z0, tr, nzf, P);
  }
  __syncthreads();
  if (!colok) return;
  const int it = __ldg(C.step);
  const bool side = min(ix - 3, nx - 4 - ix) < npd;
  const int scol = side ? xstrip_col(ix, nx, npd) : 0;
  const bool general = x0 < 3 + npd || x0 + kTileX > nx - 3 - npd || z0 < 6 || z1 - 1 > nzf - 4 ||
                       (CPML && z0 <= npd + 2) ||
                       (C.srcx >= 0 && C.srcx >= x0 - 2 && C.srcx < x0 + kTileX + 2 &&
                        C.srcz >= z0 - 2 && C.srcz < z1 + 2);
  auto cell = [&](auto gen_tag, int k) {
    constexpr bool GEN = decltype(gen_tag)::value;
    const int iz = z0 + ty + k * kTileRowStep;
    const size_t i = (size_t)iz * P + ix;
    if (k > 0) tile_load_pt<NST, NCOEF, KIND>(p, uns, accs_c, coef, nf, i);
    const bool sd = GEN && side;
    FluidTile A;
    A.init(tile, 3 + iz - z0, 4 + tx);
    const FluidCoefs cf{p.k[0], p.k[1], p.k[2], p.k[3], p.k[4], p.k[5]};
    float ade[4] = {0.f, 0.f, 0.f, 0.f}, zade[4] = {0.f, 0.f, 0.f, 0.f};
    const size_t si = (size_t)iz * C.Ps + scol;
    if (sd) {
#pragma unroll
      for (int q = 0; q < 4; ++q) ade[q] = __ldg(in.fx[q] + si);
    }
    const bool tp = GEN && CPML && iz <= npd + 2;
    const size_t zi = (size_t)(iz - 3) * P + ix;
    if (tp) {
#pragma unroll
      for (int q = 0; q < 4; ++q) zade[q] = __ldg(in.fz[q] + zi);
    }
    FluidK kk = (!GEN || (iz >= 6 && iz <= nzf - 4))
                    ? fluid_rhs<DIR, true, CPML>(C, A, iz, ix, sd, ade, cf, tp, zade)
                    : fluid_rhs<DIR, false, CPML>(C, A, iz, ix, sd, ade, cf, tp, zade);
    if (GEN) kk.p += source_term(C, iz, ix, it, s);
    const float kv[3] = {kk.vx, kk.vz, kk.p};
    float* const outs[3] = {out.fvx, out.fvz, out.fp};
    float* const accs[3] = {acc.fvx, acc.fvz, acc.fp};
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      if (KIND == kStageFirst) {
        const float u0 = A.at(f, 0, 0);
        outs[f][i] = fmaf(cc, kv[f], u0);
        accs[f][i] = fmaf(w, kv[f], u0);
      } else if (KIND == kStageMid) {
        outs[f][i] = fmaf(cc, kv[f], p.u[f]);
        accs[f][i] = fmaf(w, kv[f], p.a[f]);
      } else {
        outs[f][i] = fmaf(cc, kv[f], p.a[f]);
      }
    }
    if (sd) {
      rk_update<KIND>(kk.V0, ade[0], un.fx[0], out.fx[0], acc.fx[0], si, cc, w);
      rk_update<KIND>(kk.V1, ade[1], un.fx[1], out.fx[1], acc.fx[1], si, cc, w);
      if (kk.has_E) {
        rk_update<KIND>(kk.E0, ade[2], un.fx[2], out.fx[2], acc.fx[2], si, cc, w);
        rk_update<KIND>(kk.E1, ade[3], un.fx[3], out.fx[3], acc.fx[3], si, cc, w);
      }
    }
    if (tp) {
      rk_update<KIND>(kk.ZV0, zade[0], un.fz[0], out.fz[0], acc.fz[0], zi, cc, w);
      rk_update<KIND>(kk.ZV1, zade[1], un.fz[1], out.fz[1], acc.fz[1], zi, cc, w);
      rk_update<KIND>(kk.ZE0, zade[2], un.fz[2], out.fz[2], acc.fz[2], zi, cc, w);
      rk_update<KIND>(kk.ZE1, zade[3], un.fz[3], out.fz[3], acc.fz[3], zi, cc, w);
    }
  };
#pragma unroll 1
  for (int k = 0; k < tr / kTileRowStep; ++k) {
    if (z0 + ty + k * kTileRowStep >= z1) return;
    if (general)
      cell(std::true_type{}, k);
    else
      cell(std::false_type{}, k);
  }
}

template <int DIR, int KIND, bool CPML>
__device__ __forceinline__ void solid_tile(const Coef& C, const Fields& in, const Fields& out,
                                           const Fields& un, const Fields& acc, float cc, float w,
                                           int blk, int ntx, int tr, float* tile) {
  constexpr int NST = 5, NCOEF = 9;
  const int P = C.P, nx = C.nx, nzs = C.nzs, npd = C.npd;
  const size_t ns = (size_t)nzs * P;
  const int x0 = (blk % ntx) * kTileX, z0 = 1 + (blk / ntx) * tr;
  const int z1 = min(z0 + tr, nzs - 3);
  const int tx = threadIdx.x % kTileX, ty = threadIdx.x / kTileX;
  const int ix = x0 + tx;
  const bool colok = ix >= 3 && ix <= nx - 4;
  const float* const uns[5] = {un.svx, un.svz, un.ssx, un.ssz, un.ssxz};
  const float* const accs_c[5] = {acc.svx, acc.svz, acc.ssx, acc.ssz, acc.ssxz};
  const float* coef = C.rhos - 4 * ns;  // the solid coefficient block [9][nz_s][P]
  TilePt<NST, NCOEF> p;
  if (colok && z0 + ty < z1)
    tile_load_pt<NST, NCOEF, KIND>(p, uns, accs_c, coef, ns, (size_t)(z0 + ty) * P + ix);
  {
    const float* const f[5] = {in.svx, in.svz, in.ssx, in.ssz, in.ssxz};
    tile_stage<NST>(tile, f, x0, z0, tr, nzs, P);
  }
  __syncthreads();
  if (!colok) return;
  const bool side = min(ix - 3, nx - 4 - ix) < npd;
  const int scol = side ? xstrip_col(ix, nx, npd) : 0;
  const int zb0 = nzs - 3 - npd;  // first row of the bottom strip
  const bool general = x0 < 3 + npd || x0 + kTileX > nx - 3 - npd || z1 > zb0 || z0 < 3;
  auto cell = [&](auto gen_tag, int k) {
    constexpr bool GEN = decltype(gen_tag)::value;
    const int iz = z0 + ty + k * kTileRowStep;
    const size_t i = (size_t)iz * P + ix;
    if (k > 0) tile_load_pt<NST, NCOEF, KIND>(p, uns, accs_c, coef, ns, i);
    const bool sd = GEN && side;
    const bool bottom = GEN && iz >= zb0;
    SolidTile A;
    A.init(tile, 3 + iz - z0, 4 + tx);
    const SolidCoefs cf{p.k[0], p.k[1], p.k[2], p.k[3], p.k[4], p.k[5], p.k[6], p.k[7], p.k[8]};
    float xade[4] = {0.f, 0.f, 0.f, 0.f}, zade[4] = {0.f, 0.f, 0.f, 0.f};
    const size_t sxi = (size_t)iz * C.Ps + scol;
    const size_t szi = (size_t)(iz - zb0) * P + ix;
    if (sd) {
#pragma unroll
      for (int q = 0; q < 4; ++q) xade[q] = __ldg(in.sx[q] + sxi);
    }
    if (bottom) {
#pragma unroll
      for (int q = 0; q < 4; ++q) zade[q] = __ldg(in.sz[q] + szi);
    }
    SolidK kk = (!GEN || iz >= 3)
                    ? solid_rhs<DIR, true, CPML>(C, A, iz, ix, sd, bottom, xade, zade, cf)
                    : solid_rhs<DIR, false, CPML>(C, A, iz, ix, sd, bottom, xade, zade, cf);
    const float kv[5] = {kk.vx, kk.vz, kk.sx, kk.sz, kk.sxz};
    float* const outs[5] = {out.svx, out.svz, out.ssx, out.ssz, out.ssxz};
    float* const accs[5] = {acc.svx, acc.svz, acc.ssx, acc.ssz, acc.ssxz};
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      if (KIND == kStageFirst) {
        const float u0 = A.at(f, 0, 0);
        outs[f][i] = fmaf(cc, kv[f], u0);
        accs[f][i] = fmaf(w, kv[f], u0);
      } else if (KIND == kStageMid) {
        outs[f][i] = fmaf(cc, kv[f], p.u[f]);
        accs[f][i] = fmaf(w, kv[f], p.a[f]);
      } else {
        outs[f][i] = fmaf(cc, kv[f], p.a[f]);
      }
    }
    if (sd) {
      rk_update<KIND>(kk.XV0, xade[0], un.sx[0], out.sx[0], acc.sx[0], sxi, cc, w);
      rk_update<KIND>(kk.XV1, xade[1], un.sx[1], out.sx[1], acc.sx[1], sxi, cc, w);
      rk_update<KIND>(kk.XE0, xade[2], un.sx[2], out.sx[2], acc.sx[2], sxi, cc, w);
      rk_update<KIND>(kk.XE1, xade[3], un.sx[3], out.sx[3], acc.sx[3], sxi, cc, w);
    }
    if (bottom) {
      rk_update<KIND>(kk.ZV0, zade[0], un.sz[0], out.sz[0], acc.sz[0], szi, cc, w);
      rk_update<KIND>(kk.ZV1, zade[1], un.sz[1], out.sz[1], acc.sz[1], szi, cc, w);
      rk_update<KIND>(kk.ZE0, zade[2], un.sz[2], out.sz[2], acc.sz[2], szi, cc, w);
      rk_update<KIND>(kk.ZE1, zade[3], un.sz[3], out.sz[3], acc.sz[3], szi, cc, w);
    }
  };
#pragma unroll 1
  for (int k = 0; k < tr / kTileRowStep; ++k) {
    if (z0 + ty + k * kTileRowStep >= z1) return;
    if (general)
      cell(std::true_type{}, k);
    else
      cell(std::false_type{}, k);
  }
}

template <int DIR, int KIND, bool CPML>
__global__ void __launch_bounds__(kTileThreads, MFDM_TILE_MIN_BLOCKS)
    stage_kernel_tile(Coef C0, Fields in0, Fields out0, Fields un0, Fields acc0, int s, float cc,
                      float w, int ntx, int nbi, int nbf, int tr, int nshots) {
  __shared__ __align__(16) float tile[kTileHMax * 5 * kTileW];
  const int shot = int(blockIdx.x % unsigned(nshots));
  const int b = int(blockIdx.x / unsigned(nshots));
  const size_t so = size_t(shot) * C0.shot_stride;
  const Coef C = shot_coef(C0, shot);
  const Fields in = shot_fields(in0, so), out = shot_fields(out0, so), un = shot_fields(un0, so),
               acc = shot_fields(acc0, so);
  if (b < nbi) {
    interface_strip<DIR, KIND, CPML>(C, in, out, un, acc, cc, w, b);
  } else if (b < nbi + nbf) {
    fluid_tile<DIR, KIND, CPML>(C, in, out, un, acc, s, cc, w, b - nbi, ntx, tr, tile);
  } else {
    solid_tile<DIR, KIND, CPML>(C, in, out, un, acc, cc, w, b - nbi - nbf, ntx, tr, tile);
  }
}

// Tile height of a launch: the segment height rounded up to a multiple of 8,
// at most 48 (16 by default).
static int tile_rows_of(const Coef& C) {
  const int seg = C.seg > 0 ? C.seg : 16;
  const int tr = (seg + kTileRowStep - 1) / kTileRowStep * kTileRowStep;
  return tr < kTileRowsMax ? tr : kTileRowsMax;
}

static void tile_grid_of(int nx, int nzf, int nzs, int tr, int* ntx, int* nbf, int* nbs, int* nbi) {
  *ntx = (nx + kTileX - 1) / kTileX;
  const int frows = nzf - 1 - 3;  // fluid rows 3..nz_f-2
  const int srows = nzs - 4;      // solid rows 1..nz_s-4
  *nbf = frows > 0 ? *ntx * ((frows + tr - 1) / tr) : 0;
  *nbs = srows > 0 ? *ntx * ((srows + tr - 1) / tr) : 0;
  *nbi = (nx + kConsumers - 1) / kConsumers;
}

template <int DIR, int KIND, bool CPML>
static cudaError_t launch_tile_one(const Coef& C, const Fields& in, const Fields& out,
                                   const Fields& un, const Fields& acc, int s, cudaStream_t st) {
  int ntx, nbf, nbs, nbi;
  const int nshots = C.nshots > 0 ? C.nshots : 1, tr = tile_rows_of(C);
  tile_grid_of(C.nx, C.nzf, C.nzs, tr, &ntx, &nbf, &nbs, &nbi);
  const float cc = C.rk_c[s], w = (KIND == kStageLast) ? 0.f : C.rk_w[s];
  const unsigned grid = unsigned(nbi + nbf + nbs) * unsigned(nshots);
  stage_kernel_tile<DIR, KIND, CPML><<<grid, kTileThreads, 0, st>>>(C, in, out, un, acc, s, cc, w,
                                                                    ntx, nbi, nbf, tr, nshots);
  return cudaGetLastError();
}

template <bool CPML>
static cudaError_t launch_tile_bc(const Coef& C, const Fields& in, const Fields& out,
                                  const Fields& un, const Fields& acc, int stage, int dir,
                                  cudaStream_t st) {
  const int kind = stage == 0 ? kStageFirst : (stage == 3 ? kStageLast : kStageMid);
  if (dir == kDirF) {
    if (kind == kStageFirst) return launch_tile_one<kDirF, kStageFirst, CPML>(C, in, out, un, acc, stage, st);
    if (kind == kStageMid) return launch_tile_one<kDirF, kStageMid, CPML>(C, in, out, un, acc, stage, st);
    return launch_tile_one<kDirF, kStageLast, CPML>(C, in, out, un, acc, stage, st);
  }
  if (kind == kStageFirst) return launch_tile_one<kDirB, kStageFirst, CPML>(C, in, out, un, acc, stage, st);
  if (kind == kStageMid) return launch_tile_one<kDirB, kStageMid, CPML>(C, in, out, un, acc, stage, st);
  return launch_tile_one<kDirB, kStageLast, CPML>(C, in, out, un, acc, stage, st);
}

cudaError_t launch_stage_tile(const Coef& C, const Fields& in, const Fields& out, const Fields& un,
                              const Fields& acc, int stage, int dir, cudaStream_t st) {
  return C.cpml ? launch_tile_bc<true>(C, in, out, un, acc, stage, dir, st)
                : launch_tile_bc<false>(C, in, out, un, acc, stage, dir, st);
}

#endif  // MFDM_VARIANT_TU

}  // namespace MFDM_VNS

#ifndef MFDM_VARIANT_TU
// ---- built once: the finish kernel, small kernels and the dispatching launchers ----

namespace v3 {
cudaError_t configure();
cudaError_t launch_stage_v(const Coef& C, const Fields& in, const Fields& out, const Fields& un,
                           const Fields& acc, const StageMaps& maps, int stage, int dir,
                           cudaStream_t st);
cudaError_t upload_constants_v(const float* srcw25, const float* w7);
}  // namespace v3

constexpr int kFinishThreads = 256;  // filter / receiver kernel

// Post-step interface filter (7-point Gaussian along x, renormalised at the
// clamped ends) and continuity average (src/pml_fs_kernels.cu:428-525),
// evaluated out of place from C.ipre, so no block reads values another block
// already filtered. Then the receiver rows are sampled (src/main.cu:195-211)
// and the last block to finish advances the device step counter.
__global__ void __launch_bounds__(kFinishThreads) finish_kernel(Coef C0, Fields U0) {
  const Coef C = shot_coef(C0, blockIdx.y);
  const Fields U = shot_fields(U0, size_t(blockIdx.y) * C0.shot_stride);
  const int nx = C.nx, P = C.P, nzf = C.nzf;
  const int ix = blockIdx.x * kFinishThreads + threadIdx.x;
  const int it = *C.step;
  float r0 = 0.f, r1 = 0.f, r2 = 0.f;
  if (ix >= 3 && ix <= nx - 4) {
    const int klo = max(-3, 3 - ix), khi = min(3, nx - 4 - ix);
    // taps k = klo..khi in ascending order (the reference's summation order);
    // fully unrolled and predicated, so all loads are in flight together
    float wsum = 0.0f;
#pragma unroll
    for (int k = -3; k <= 3; ++k)
      if (k >= klo && k <= khi) wsum += c_w7[k + 3];
    float v[8];
#pragma unroll
    for (int f = 0; f < 8; ++f) {
      float t[7];
#pragma unroll
      for (int k = -3; k <= 3; ++k)
        t[k + 3] = (k >= klo && k <= khi) ? __ldg(C.ipre + (size_t)f * P + ix + k) : 0.f;
      float sum = 0.0f;
#pragma unroll
      for (int k = -3; k <= 3; ++k)
        if (k >= klo && k <= khi) sum += c_w7[k + 3] * t[k + 3];
      v[f] = sum / wsum;
    }
    float u[8];
    interface_average(__ldg(C.nrm + ix), v, u);
    const size_t fi = (size_t)(nzf - 1) * P + ix;
    U.fvx[fi] = u[0];
    U.fvz[fi] = u[1];
    U.fp[fi] = u[2];
    r0 = u[3];
    r1 = u[4];
    r2 = u[2];
    U.svx[ix] = u[3];
    U.svz[ix] = u[4];
    U.ssx[ix] = u[5];
    U.ssz[ix] = u[6];
    U.ssxz[ix] = u[7];
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
    if (prev == gridDim.x * gridDim.y - 1) {
      *C.done = 0u;
      *C.step = it + 1;
      __threadfence();
    }
  }
}

__global__ void reciprocal_rows_kernel(float* a, int rows, int nx, int P) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x, iz = blockIdx.y;
  if (ix < nx && iz < rows) {
    float* p = a + (size_t)iz * P + ix;
    *p = float(1.0 / double(*p));
  }
}

__global__ void set_step_kernel(int* step, unsigned* done, int it) {
  *step = it;
  *done = 0u;
}

// ---- host-side launchers ------------------------------------------------------

size_t stage_smem_bytes() { return v2::smem_bytes(); }

int stage_seg_rows(const Coef& C) { return C.seg > 0 ? C.seg : default_seg_rows(C); }

void stage_grid(int nx, int nzf, int nzs, int seg, int* ntx, int* nbf, int* nbs, int* nbi) {
  v2::grid_of(nx, nzf, nzs, seg, ntx, nbf, nbs, nbi);
}

int stage_blocks_per_sm(const Coef& C) {
  if (C.variant == 2 || C.variant == 3 || C.variant == 4) return C.variant;
  // with the default segment heights the 3-block build is the fastest at
  // 4096x2048 (24 rows), 2048x1024 and 1200x800 (8 rows)
  return 3;
}

cudaError_t configure_device() {
  const cudaError_t e = v2::configure();
  return e != cudaSuccess ? e : v3::configure();
}

cudaError_t launch_stage(const Coef& C, const Fields& in, const Fields& out, const Fields& un,
                         const Fields& acc, const StageMaps& maps, int stage, int dir,
                         cudaStream_t st) {
  const int v = stage_blocks_per_sm(C);
  if (v == 4) return v2::launch_stage_tile(C, in, out, un, acc, stage, dir, st);
  return v == 3 ? v3::launch_stage_v(C, in, out, un, acc, maps, stage, dir, st)
                : v2::launch_stage_v(C, in, out, un, acc, maps, stage, dir, st);
}

cudaError_t launch_finish(const Coef& C, const Fields& U, cudaStream_t st) {
  const int nb = (C.nx + kFinishThreads - 1) / kFinishThreads;
  finish_kernel<<<dim3(unsigned(nb), unsigned(C.nshots > 0 ? C.nshots : 1)), kFinishThreads, 0, st>>>(C, U);
  return cudaGetLastError();
}

cudaError_t launch_reciprocal(float* a, int rows, int nx, int P, cudaStream_t st) {
  if (rows <= 0 || nx <= 0) return cudaSuccess;
  reciprocal_rows_kernel<<<dim3((nx + 255) / 256, rows), 256, 0, st>>>(a, rows, nx, P);
  return cudaGetLastError();
}

cudaError_t launch_set_step(const Coef& C, int it, cudaStream_t st) {
  set_step_kernel<<<1, 1, 0, st>>>(C.step, C.done, it);
  return cudaGetLastError();
}

cudaError_t upload_constants(const float* srcw25, const float* w7) {
  cudaError_t e = cudaMemcpyToSymbol(c_srcw, srcw25, 25 * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_w7, w7, 7 * sizeof(float));
  if (e == cudaSuccess) e = v2::upload_constants_v(srcw25, w7);
  return e != cudaSuccess ? e : v3::upload_constants_v(srcw25, w7);
}

#endif  // MFDM_VARIANT_TU

}  // namespace mfdm
