// CPU oracle for the MarineSeis-FDM-2D fluid-solid time step (FANDS with
// boundary type PANDF, and with CPML: CFS-PML on all four sides).
//
// TEST INFRASTRUCTURE ONLY. This file restates, on the CPU, the reference
// algorithm of `PmlFs::FluidSolid::update_RK4` so that the CUDA library can be
// checked against it. Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / reference legs load it; the product library never does.
//
// Precision: templated on the arithmetic type. With `float` every expression
// is evaluated in the same order as the reference source (no FMA contraction:
// compile with -ffp-contract=off), so it reproduces the reference's FP32
// arithmetic up to the FMA contraction nvcc applies on the GPU. With `double`
// the same discrete operator (the same float-valued stencil, filter and source
// weights) is evaluated in FP64: it is the FP64 oracle that FP32 results are
// measured against.
//
// Reference files followed (paths inside the reference project):
//   include/tools_func.cuh:6-188, src/tools_func.cu:10-65  operators, fluxes, ghost reads
//   include/pml_fs_kernels.cuh:333-827                     RHS kernels, interface projection
//   src/pml_fs_kernels.cu:385-531, 624-868                 ghosts, filter, source, RK4 driver
//   src/elements.cu:18-40, 121-124, 385-392, 824-905       constants, CFS shape, Ricker, PML tables, normals
//   src/main.cu:92, 136-213, 245-295                       step loop and record sampling
//   include/cpml_kernels.cuh:237-662                       the CPML variant (Cpml::FluidSolid):
//       fluid without a free surface, a top zeta-PML band in the fluid, and the
//       solid sxz read with the solid-local index into the global metric (:448-455)
//
// One deliberate difference: the interface filter (src/pml_fs_kernels.cu:428-525)
// runs in place in the reference, so a block may read a neighbour's halo after
// that neighbour already stored filtered values. The oracle filters out of
// place (every read sees the unfiltered row), which is the race-free reading.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>
#include <xmmintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// DRP-optimised biased first derivative, taps -1..+3 (include/tools_func.cuh:6-10).
constexpr float kAm1 = -0.30874f;
constexpr float kA0 = -0.63260f;
constexpr float kA1 = +1.23300f;
constexpr float kA2 = -0.33340f;
constexpr float kA3 = +0.04168f;
// 4-2 and 2-2 one-sided operators (include/tools_func.cuh:12-17).
constexpr float kM42_0 = -7.0f / 6.0f;
constexpr float kM42_1 = +8.0f / 6.0f;
constexpr float kM42_2 = -1.0f / 6.0f;
constexpr float kM22_0 = -1.0f;
constexpr float kM22_1 = +1.0f;
// Interface-row 7-point Gaussian (src/elements.cu:30-33).
constexpr float kW7[7] = {1.1e-13f, 1.678e-06f, 0.03419f, 0.93163f,
                          0.03419f, 1.678e-06f, 1.1e-13f};
// 5x5 source spreading weights (src/elements.cu:34-40).
constexpr float kSrcW[5][5] = {
    {0.0030f, 0.0133f, 0.0219f, 0.0133f, 0.0030f},
    {0.0133f, 0.0596f, 0.0983f, 0.0596f, 0.0133f},
    {0.0219f, 0.0983f, 0.1621f, 0.0983f, 0.0219f},
    {0.0133f, 0.0596f, 0.0983f, 0.0596f, 0.0133f},
    {0.0030f, 0.0133f, 0.0219f, 0.0133f, 0.0030f}};

enum Dir { kF = 0, kB = 1 };

// Field slots of one RK state set. Fluid-sized: 0..2 and 8..11; solid-sized: the rest.
enum Field {
  FVX, FVZ, FP,                // fluid velocity, pressure
  SVX, SVZ, SSX, SSZ, SSXZ,    // solid velocity, stress
  FXVX, FXVZ, FXEX, FXEZ,      // fluid xi-ADE memory
  SXVX, SXVZ, SXEX, SXEZ,      // solid xi-ADE memory
  SZVX, SZVZ, SZEX, SZEZ,      // solid zeta-ADE memory
  FZVX, FZVZ, FZEX, FZEZ,      // fluid zeta-ADE memory (top band, CPML only)
  NFIELD
};
inline bool is_fluid(int f) { return f <= FP || (f >= FXVX && f <= FXEZ) || f >= FZVX; }

template <class R> struct P2 { R x, y; };

// Biased 5-point derivative along a stride (include/tools_func.cuh:50-92).
template <class R>
inline R dmac(int dir, const R* f, std::ptrdiff_t s) {
  if (dir == kF)
    return R(kAm1) * f[-s] + R(kA0) * f[0] + R(kA1) * f[s] + R(kA2) * f[2 * s] +
           R(kA3) * f[3 * s];
  return -R(kAm1) * f[s] - R(kA0) * f[0] - R(kA1) * f[-s] - R(kA2) * f[-2 * s] -
         R(kA3) * f[-3 * s];
}

// Order-reduced zeta derivative by distance to a boundary (include/tools_func.cuh:94-140).
template <class R>
inline R dz_near(int dir, const R* f, std::ptrdiff_t s, int dist, bool solid_side) {
  if (dist >= 3) return dmac(dir, f, s);
  if (dist == 2) {
    if (dir == kF) return R(kM42_0) * f[0] + R(kM42_1) * f[s] + R(kM42_2) * f[2 * s];
    return -R(kM42_0) * f[0] - R(kM42_1) * f[-s] - R(kM42_2) * f[-2 * s];
  }
  int d = dir;
  if (dist <= 0) d = solid_side ? kF : kB;
  if (d == kF) return R(kM22_0) * f[0] + R(kM22_1) * f[s];
  return -R(kM22_0) * f[0] - R(kM22_1) * f[-s];
}

// The same biased derivative applied to a two-component flux (include/tools_func.cuh:142-188).
template <class R, class Fn>
inline P2<R> dflux(int dir, Fn F) {
  P2<R> o;
  if (dir == kF) {
    P2<R> m1 = F(-1), c0 = F(0), p1 = F(1), p2 = F(2), p3 = F(3);
    o.x = R(kAm1) * m1.x + R(kA0) * c0.x + R(kA1) * p1.x + R(kA2) * p2.x + R(kA3) * p3.x;
    o.y = R(kAm1) * m1.y + R(kA0) * c0.y + R(kA1) * p1.y + R(kA2) * p2.y + R(kA3) * p3.y;
  } else {
    P2<R> p1 = F(1), c0 = F(0), m1 = F(-1), m2 = F(-2), m3 = F(-3);
    o.x = -(R(kAm1) * p1.x + R(kA0) * c0.x + R(kA1) * m1.x + R(kA2) * m2.x + R(kA3) * m3.x);
    o.y = -(R(kAm1) * p1.y + R(kA0) * c0.y + R(kA1) * m1.y + R(kA2) * m2.y + R(kA3) * m3.y);
  }
  return o;
}

}  // namespace

extern "C" {
// Model description handed in from Python (ctypes). All arrays are row-major
// [rows][nx] doubles; the FP32 oracle rounds them to float first.
struct orc_model {
  int nx, nz_f, nz_s;  // fluid and solid row counts, both including the interface row
  int npd, npow;
  double fpeak, dt, thickness, vp_max, rc, beta0;
  int src_x, src_z;    // source column and fluid row
  const double *K, *rho_f;                          // [nz_f][nx]
  const double *C11, *C13, *C33, *C55, *rho_s;      // [nz_s][nx]
  const double *J, *xi_x, *xi_z, *ze_x, *ze_z;      // [nz_f + nz_s - 1][nx]
  int cpml;            // 1: CFS-PML on all four sides (boundary type CPML), 0: PANDF
};
}

namespace {

// CFS-PML 1-D profile over n cells with a band of npd cells at the low and/or
// high end (src/elements.cu:824-860): d = d0 r^NPOW, beta = 1 + (beta0 - 1) r^2,
// alpha = alpha0 (1 - r), r = k / npd. The FP32 oracle evaluates it with float
// std::log / std::pow like the reference; the FP64 oracle in double from the
// float-valued inputs.
template <class R>
void pml_profile(const orc_model& m, float fpeak_f, int npd, R* al, R* be, R* dp, int n, bool lo,
                 bool hi) {
  const float vpmax = float(m.vp_max), rc = float(m.rc), thick = float(m.thickness);
  const float beta0 = float(m.beta0);
  const int npow = m.npow;
  const float alpha0_f = 2 * float(M_PI) * fpeak_f;
  const float damp0_f = -(npow + 1) * vpmax * std::log(rc) / (2.0f * thick);
  const double alpha0_d = 2.0 * M_PI * double(fpeak_f);
  const double damp0_d = -(npow + 1) * double(vpmax) * std::log(double(rc)) / (2.0 * double(thick));
  for (int i = 0; i < n; ++i) {
    int k = -1;
    if (lo && i >= 3 && i <= 2 + npd) k = 3 + npd - i;
    if (hi && i >= n - 3 - npd && i <= n - 4) k = i - (n - 4 - npd);
    if constexpr (std::is_same<R, float>::value) {
      if (k <= 0) { dp[i] = 0.0f; be[i] = 1.0f; al[i] = alpha0_f; }
      else {
        float r = float(k) / float(npd);
        dp[i] = damp0_f * std::pow(r, float(npow));
        be[i] = 1.0f + (beta0 - 1.0f) * std::pow(r, 2.0f);
        al[i] = alpha0_f * (1.0f - std::pow(r, 1.0f));
      }
    } else {
      if (k <= 0) { dp[i] = 0.0; be[i] = 1.0; al[i] = R(alpha0_d); }
      else {
        double r = double(k) / double(npd);
        dp[i] = R(damp0_d * std::pow(r, double(npow)));
        be[i] = R(1.0 + (double(beta0) - 1.0) * r * r);
        al[i] = R(alpha0_d * (1.0 - r));
      }
    }
  }
}

template <class R>
struct Oracle {
  int nx, nzf, nzs, npd;
  bool cpml;
  float fpeak_f, dt_f;
  int srcx, srcz;
  std::vector<R> K, rf, C11, C13, C33, C55, rs, J, xx, xz, zx, zz;
  std::vector<R> alx, bex, dpx, alz, bez, dpz;  // xi tables [nx], solid zeta tables [nzs]
  std::vector<R> alzf, bezf, dpzf;              // fluid zeta tables [nzf] (top band, CPML)
  std::vector<R> nfx, nfz;                      // interface normal [nx]
  using Set = std::vector<std::vector<R>>;
  Set U, Ub, Ut, Kk;
  std::vector<P2<R>> Gf, Gs, Gfs;

  static std::vector<R> conv(const double* p, size_t n) {
    std::vector<R> v(n);
    for (size_t i = 0; i < n; ++i) {
      if constexpr (std::is_same<R, float>::value) v[i] = float(p[i]);
      else v[i] = p[i];
    }
    return v;
  }

  void alloc(Set& s) {
    s.assign(NFIELD, {});
    for (int f = 0; f < NFIELD; ++f) s[f].assign(size_t(is_fluid(f) ? nzf : nzs) * nx, R(0));
  }

  explicit Oracle(const orc_model& m) {
    nx = m.nx; nzf = m.nz_f; nzs = m.nz_s; npd = m.npd;
    cpml = m.cpml != 0;
    fpeak_f = float(m.fpeak); dt_f = float(m.dt);
    srcx = m.src_x; srcz = m.src_z;
    const size_t nf = size_t(nzf) * nx, ns = size_t(nzs) * nx, ng = size_t(nzf + nzs - 1) * nx;
    K = conv(m.K, nf); rf = conv(m.rho_f, nf);
    C11 = conv(m.C11, ns); C13 = conv(m.C13, ns); C33 = conv(m.C33, ns); C55 = conv(m.C55, ns);
    rs = conv(m.rho_s, ns);
    J = conv(m.J, ng); xx = conv(m.xi_x, ng); xz = conv(m.xi_z, ng);
    zx = conv(m.ze_x, ng); zz = conv(m.ze_z, ng);
    pml_tables(m);
    normals();
    alloc(U); alloc(Ub); alloc(Ut); alloc(Kk);
    Gf.assign(3 * nx, {R(0), R(0)}); Gs = Gf; Gfs = Gf;
    build_jobs();
  }

  // CFS-PML 1-D profiles (src/elements.cu:121-124, 824-873). The FP32 oracle
  // evaluates them with float std::log/std::pow like the reference; the FP64
  // oracle evaluates the same formulas in double from the float-valued inputs.
  void pml_tables(const orc_model& m) {
    alx.assign(nx, 0); bex.assign(nx, 0); dpx.assign(nx, 0);
    alz.assign(nzs, 0); bez.assign(nzs, 0); dpz.assign(nzs, 0);
    alzf.assign(nzf, 0); bezf.assign(nzf, 0); dpzf.assign(nzf, 0);
    pml_profile(m, fpeak_f, npd, alx.data(), bex.data(), dpx.data(), nx, true, true);
    pml_profile(m, fpeak_f, npd, alz.data(), bez.data(), dpz.data(), nzs, false, true);
    // fluid zeta axis: a top band for CPML only (src/elements.cu:866-869)
    pml_profile(m, fpeak_f, npd, alzf.data(), bezf.data(), dpzf.data(), nzf, cpml, false);
  }

  // Unit normal of the interface from the zeta gradient (src/elements.cu:892-905).
  void normals() {
    nfx.assign(nx, 0); nfz.assign(nx, 0);
    const size_t row = size_t(nzf - 1) * nx;
    for (int ix = 0; ix < nx; ++ix) {
      R a = zx[row + ix], b = zz[row + ix];
      R s = std::sqrt(a * a + b * b);
      nfx[ix] = a / s; nfz[ix] = b / s;
    }
  }

  // Ricker wavelet at stage time t (src/elements.cu:385-392).
  R ricker(R time) const {
    if constexpr (std::is_same<R, float>::value) {
      const float T = float(1.2 / double(fpeak_f));
      float t = float(time) - T;
      if (t > T) return 0.0f;
      float temp = float(M_PI * double(fpeak_f) * double(t));
      temp *= temp;
      return (1 - 2 * temp) * std::exp(-temp);
    }
    const double T = 1.2 / double(fpeak_f);
    double t = double(time) - T;
    if (t > T) return 0.0;
    double temp = M_PI * double(fpeak_f) * t;
    temp *= temp;
    return R((1 - 2 * temp) * std::exp(-temp));
  }

  // ---- fluxes (src/tools_func.cu:19-65) ----
  P2<R> flux_ze_f(const Set& S, int r, int ix) const {
    size_t i = size_t(r) * nx + ix;
    return {-J[i] * zx[i] * S[FP][i], -J[i] * zz[i] * S[FP][i]};
  }
  P2<R> flux_xi_f(const Set& S, size_t i) const {
    return {-J[i] * xx[i] * S[FP][i], -J[i] * xz[i] * S[FP][i]};
  }
  P2<R> flux_ze_s(const Set& S, int r, int ix) const {
    size_t i = size_t(r) * nx + ix, g = i + size_t(nzf - 1) * nx;
    return {J[g] * (zx[g] * S[SSX][i] + zz[g] * S[SSXZ][i]),
            J[g] * (zx[g] * S[SSXZ][i] + zz[g] * S[SSZ][i])};
  }
  P2<R> flux_xi_s(const Set& S, size_t i) const {
    size_t g = i + size_t(nzf - 1) * nx;
    return {J[g] * (xx[g] * S[SSX][i] + xz[g] * S[SSXZ][i]),
            J[g] * (xx[g] * S[SSXZ][i] + xz[g] * S[SSZ][i])};
  }

  // Mirrored ghost fluxes beside the interface and the free surface (src/pml_fs_kernels.cu:385-426).
  void build_ghosts(const Set& S) {
    for (int ix = 3; ix <= nx - 4; ++ix) {
      P2<R> f0 = flux_ze_f(S, nzf - 1, ix);
      P2<R> s0 = flux_ze_s(S, 0, ix);
      for (int n = 1; n <= 3; ++n) {
        P2<R> fn = flux_ze_f(S, nzf - 1 - n, ix);
        Gf[(n - 1) * nx + ix] = {2 * f0.x - fn.x, 2 * f0.y - fn.y};
        P2<R> sn = flux_ze_s(S, n, ix);
        Gs[(n - 1) * nx + ix] = {2 * s0.x - sn.x, 2 * s0.y - sn.y};
        P2<R> gn = flux_ze_f(S, 3 + n, ix);
        Gfs[(n - 1) * nx + ix] = {-gn.x, -gn.y};
      }
    }
  }

  // Fluid momentum RHS (include/pml_fs_kernels.cuh:333-450; CPML:
  // include/cpml_kernels.cuh:240-342 - no free-surface rows, a top zeta band).
  void fluid_velocity(int dir, const Set& S) {
#pragma omp parallel for schedule(static)
    for (int iz = 3; iz < nzf; ++iz) {
      for (int ix = 3; ix <= nx - 4; ++ix) {
        const size_t i = size_t(iz) * nx + ix;
        const R xix = xx[i], xiz = xz[i], zex = zx[i], zez = zz[i];
        const R gxx = xix * xix + xiz * xiz;
        const R gzz = zex * zex + zez * zez;
        const bool top = cpml && iz <= npd + 2;
        R rvx, rvz, divx, divz, divzx = 0, divzz = 0;
        const int d_if = nzf - 1 - iz, d_fs = cpml ? 3 : iz - 3;
        if (d_if < 3 || d_fs < 3) {
          auto Fxi = [&](int j) { return flux_xi_f(S, i + j); };
          auto Fze = [&](int j) -> P2<R> {
            int r = iz + j;
            if (d_if < 3) {
              if (r <= nzf - 1) return flux_ze_f(S, r, ix);
              return Gf[size_t(r - nzf) * nx + ix];
            }
            if (r >= 3) return flux_ze_f(S, r, ix);
            return Gfs[size_t(2 - r) * nx + ix];
          };
          P2<R> a = dflux<R>(dir, Fxi), b = dflux<R>(dir, Fze);
          const R Sx = a.x + b.x, Sz = a.y + b.y, Jc = J[i];
          rvx = Sx / Jc;
          rvz = Sz / Jc;
          divx = xix * (xix * Sx + xiz * Sz) / (gxx * Jc);
          divz = xiz * (xix * Sx + xiz * Sz) / (gxx * Jc);
          if (top) {
            divzx = zex * (zex * Sx + zez * Sz) / (gzz * Jc);
            divzz = zez * (zex * Sx + zez * Sz) / (gzz * Jc);
          }
        } else {
          const R dpdx = dmac(dir, &S[FP][i], 1), dpdz = dmac(dir, &S[FP][i], nx);
          rvx = -(xix * dpdx + zex * dpdz);
          rvz = -(xiz * dpdx + zez * dpdz);
          const R gxz = xix * zex + xiz * zez;
          divx = -xix * (gxx * dpdx + gxz * dpdz) / gxx;
          divz = -xiz * (gxx * dpdx + gxz * dpdz) / gxx;
          if (top) {
            divzx = -zex * (gxz * dpdx + gzz * dpdz) / gzz;
            divzz = -zez * (gxz * dpdx + gzz * dpdz) / gzz;
          }
        }
        const R rho = rf[i];
        R kvx = rvx / rho, kvz = rvz / rho;
        const int distx = std::min(ix - 3, nx - 4 - ix);
        if (distx < npd) {
          const R dpb = dpx[ix] / bex[ix], apdpb = alx[ix] + dpb, invb = R(1) / bex[ix];
          const R V0 = S[FXVX][i], V1 = S[FXVZ][i];
          Kk[FXVX][i] = -apdpb * V0 + dpb * divx;
          Kk[FXVZ][i] = -apdpb * V1 + dpb * divz;
          kvx += ((invb - R(1)) * divx - invb * V0) / rho;
          kvz += ((invb - R(1)) * divz - invb * V1) / rho;
        }
        if (top) {
          const R dpb = dpzf[iz] / bezf[iz], apdpb = alzf[iz] + dpb, invb = R(1) / bezf[iz];
          const R V0 = S[FZVX][i], V1 = S[FZVZ][i];
          Kk[FZVX][i] = -apdpb * V0 + dpb * divzx;
          Kk[FZVZ][i] = -apdpb * V1 + dpb * divzz;
          kvx += ((invb - R(1)) * divzx - invb * V0) / rho;
          kvz += ((invb - R(1)) * divzz - invb * V1) / rho;
        }
        Kk[FVX][i] = kvx;
        Kk[FVZ][i] = kvz;
      }
    }
  }

  // Fluid pressure RHS (include/pml_fs_kernels.cuh:452-507; CPML:
  // include/cpml_kernels.cuh:345-415 - row 3 is an ordinary row, a top zeta band).
  void fluid_stress(int dir, const Set& S) {
#pragma omp parallel for schedule(static)
    for (int iz = 3; iz < nzf; ++iz) {
      for (int ix = 3; ix <= nx - 4; ++ix) {
        const size_t i = size_t(iz) * nx + ix;
        if (!cpml && iz == 3) { Kk[FP][i] = 0; continue; }
        const R xix = xx[i], xiz = xz[i], zex = zx[i], zez = zz[i];
        const R dvxdx = dmac(dir, &S[FVX][i], 1), dvzdx = dmac(dir, &S[FVZ][i], 1);
        const int dn = cpml ? nzf - 1 - iz : std::min(iz - 3, nzf - 1 - iz);
        const R dvxdz = dz_near(dir, &S[FVX][i], nx, dn, false);
        const R dvzdz = dz_near(dir, &S[FVZ][i], nx, dn, false);
        const R Kc = K[i];
        R kp = -Kc * (xix * dvxdx + zex * dvxdz + xiz * dvzdx + zez * dvzdz);
        const int distx = std::min(ix - 3, nx - 4 - ix);
        if (distx < npd) {
          const R gxx = xix * xix + xiz * xiz, gxz = xix * zex + xiz * zez;
          const R Dvx = dvxdx + (gxz / gxx) * dvxdz, Dvz = dvzdx + (gxz / gxx) * dvzdz;
          const R dpb = dpx[ix] / bex[ix], apdpb = alx[ix] + dpb, invb = R(1) / bex[ix];
          const R E0 = S[FXEX][i], E1 = S[FXEZ][i];
          Kk[FXEX][i] = -apdpb * E0 + dpb * Dvx;
          Kk[FXEZ][i] = -apdpb * E1 + dpb * Dvz;
          if (cpml)
            kp += -Kc * (invb - R(1)) * xix * Dvx - Kc * (invb - R(1)) * xiz * Dvz +
                  invb * Kc * xix * E0 + invb * Kc * xiz * E1;
          else
            kp += Kc * (-(invb - R(1)) * xix * Dvx - (invb - R(1)) * xiz * Dvz +
                        invb * xix * E0 + invb * xiz * E1);
        }
        if (cpml && iz <= npd + 2) {
          const R gxz = xix * zex + xiz * zez, gzz = zex * zex + zez * zez;
          const R Dzx = dvxdz + (gxz / gzz) * dvxdx, Dzz = dvzdz + (gxz / gzz) * dvzdx;
          const R dpb = dpzf[iz] / bezf[iz], apdpb = alzf[iz] + dpb, invb = R(1) / bezf[iz];
          const R E0 = S[FZEX][i], E1 = S[FZEZ][i];
          Kk[FZEX][i] = -apdpb * E0 + dpb * Dzx;
          Kk[FZEZ][i] = -apdpb * E1 + dpb * Dzz;
          kp += Kc * (-(invb - R(1)) * (zex * Dzx + zez * Dzz) + invb * (zex * E0 + zez * E1));
        }
        Kk[FP][i] = kp;
      }
    }
  }

  // Solid stress RHS, VTI law (include/pml_fs_kernels.cuh:509-628).
  void solid_stress(int dir, const Set& S) {
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nzs - 3; ++iz) {
      for (int ix = 3; ix <= nx - 4; ++ix) {
        const size_t i = size_t(iz) * nx + ix, g = i + size_t(nzf - 1) * nx;
        const R xix = xx[g], xiz = xz[g], zex = zx[g], zez = zz[g];
        const R dvxdx = dmac(dir, &S[SVX][i], 1);
        const R dvxdz = dz_near(dir, &S[SVX][i], nx, iz, true);
        const R dvzdx = dmac(dir, &S[SVZ][i], 1);
        const R dvzdz = dz_near(dir, &S[SVZ][i], nx, iz, true);
        const R c11 = C11[i], c13 = C13[i], c33 = C33[i], c55 = C55[i];
        R ksx = c11 * (xix * dvxdx + zex * dvxdz) + c13 * (xiz * dvzdx + zez * dvzdz);
        R ksz = c13 * (xix * dvxdx + zex * dvxdz) + c33 * (xiz * dvzdx + zez * dvzdz);
        // CPML reads this line's metric with the solid-local index i, i.e. at
        // global row iz (include/cpml_kernels.cuh:448-455); kept for parity.
        R ksxz = cpml ? c55 * (xz[i] * dvxdx + zz[i] * dvxdz + xx[i] * dvzdx + zx[i] * dvzdz)
                      : c55 * (xiz * dvxdx + zez * dvxdz + xix * dvzdx + zex * dvzdz);
        const int distx = std::min(ix - 3, nx - 4 - ix);
        const bool side = distx < npd, bottom = iz >= nzs - 3 - npd;
        if (side || bottom) {
          const R gxx = xix * xix + xiz * xiz, gxz = xix * zex + xiz * zez,
                  gzz = zex * zex + zez * zez;
          if (side) {
            const R Dvx = dvxdx + (gxz / gxx) * dvxdz, Dvz = dvzdx + (gxz / gxx) * dvzdz;
            const R dpb = dpx[ix] / bex[ix], apdpb = alx[ix] + dpb, invb = R(1) / bex[ix];
            const R E0 = S[SXEX][i], E1 = S[SXEZ][i];
            Kk[SXEX][i] = -apdpb * E0 + dpb * Dvx;
            Kk[SXEZ][i] = -apdpb * E1 + dpb * Dvz;
            ksx += c11 * (invb - R(1)) * xix * Dvx + c13 * (invb - R(1)) * xiz * Dvz -
                   invb * c11 * xix * E0 - invb * c13 * xiz * E1;
            ksz += c13 * (invb - R(1)) * xix * Dvx + c33 * (invb - R(1)) * xiz * Dvz -
                   invb * c13 * xix * E0 - invb * c33 * xiz * E1;
            ksxz += c55 * (invb - R(1)) * (xiz * Dvx + xix * Dvz) - invb * c55 * xiz * E0 -
                    invb * c55 * xix * E1;
          }
          if (bottom) {
            const R Dvx = dvxdz + (gxz / gzz) * dvxdx, Dvz = dvzdz + (gxz / gzz) * dvzdx;
            const R dpb = dpz[iz] / bez[iz], apdpb = alz[iz] + dpb, invb = R(1) / bez[iz];
            const R E0 = S[SZEX][i], E1 = S[SZEZ][i];
            Kk[SZEX][i] = -apdpb * E0 + dpb * Dvx;
            Kk[SZEZ][i] = -apdpb * E1 + dpb * Dvz;
            ksx += c11 * (invb - R(1)) * zex * Dvx + c13 * (invb - R(1)) * zez * Dvz -
                   invb * c11 * zex * E0 - invb * c13 * zez * E1;
            ksz += c13 * (invb - R(1)) * zex * Dvx + c33 * (invb - R(1)) * zez * Dvz -
                   invb * c13 * zex * E0 - invb * c33 * zez * E1;
            ksxz += c55 * (invb - R(1)) * (zez * Dvx + zex * Dvz) - invb * c55 * zez * E0 -
                    invb * c55 * zex * E1;
          }
        }
        Kk[SSX][i] = ksx;
        Kk[SSZ][i] = ksz;
        Kk[SSXZ][i] = ksxz;
      }
    }
  }

  // Solid momentum RHS (include/pml_fs_kernels.cuh:631-752).
  void solid_velocity(int dir, const Set& S) {
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nzs - 3; ++iz) {
      for (int ix = 3; ix <= nx - 4; ++ix) {
        const size_t i = size_t(iz) * nx + ix, g = i + size_t(nzf - 1) * nx;
        const R xix = xx[g], xiz = xz[g], zex = zx[g], zez = zz[g];
        const R gxx = xix * xix + xiz * xiz, gzz = zex * zex + zez * zez;
        R rvx, rvz, dxx, dxz, dzx, dzz;
        if (iz < 3) {
          auto Fxi = [&](int j) { return flux_xi_s(S, i + j); };
          auto Fze = [&](int j) -> P2<R> {
            int r = iz + j;
            if (r >= 0) return flux_ze_s(S, r, ix);
            return Gs[size_t(-r - 1) * nx + ix];
          };
          P2<R> a = dflux<R>(dir, Fxi), b = dflux<R>(dir, Fze);
          const R Sx = a.x + b.x, Sz = a.y + b.y, Jc = J[g];
          rvx = Sx / Jc;
          rvz = Sz / Jc;
          dxx = xix * (xix * Sx + xiz * Sz) / (gxx * Jc);
          dxz = xiz * (xix * Sx + xiz * Sz) / (gxx * Jc);
          dzx = zex * (zex * Sx + zez * Sz) / (gzz * Jc);
          dzz = zez * (zex * Sx + zez * Sz) / (gzz * Jc);
        } else {
          const R sxdx = dmac(dir, &S[SSX][i], 1), sxdz = dmac(dir, &S[SSX][i], nx);
          const R szdx = dmac(dir, &S[SSZ][i], 1), szdz = dmac(dir, &S[SSZ][i], nx);
          const R tdx = dmac(dir, &S[SSXZ][i], 1), tdz = dmac(dir, &S[SSXZ][i], nx);
          rvx = xix * sxdx + zex * sxdz + xiz * tdx + zez * tdz;
          rvz = xix * tdx + zex * tdz + xiz * szdx + zez * szdz;
          const R gxz = xix * zex + xiz * zez;
          dxx = xix * (sxdx + gxz / gxx * sxdz) + xiz * (tdx + gxz / gxx * tdz);
          dxz = xix * (tdx + gxz / gxx * tdz) + xiz * (szdx + gxz / gxx * szdz);
          dzx = zex * (sxdz + gxz / gzz * sxdx) + zez * (gxz / gzz * tdx + tdz);
          dzz = zex * (gxz / gzz * tdx + tdz) + zez * (gxz / gzz * szdx + szdz);
        }
        const int distx = std::min(ix - 3, nx - 4 - ix);
        const bool side = distx < npd, bottom = iz >= nzs - 3 - npd;
        const R rho = rs[i];
        R kvx = rvx / rho, kvz = rvz / rho;
        if (side) {
          const R dpb = dpx[ix] / bex[ix], apdpb = alx[ix] + dpb, invb = R(1) / bex[ix];
          const R V0 = S[SXVX][i], V1 = S[SXVZ][i];
          Kk[SXVX][i] = -apdpb * V0 + dpb * dxx;
          Kk[SXVZ][i] = -apdpb * V1 + dpb * dxz;
          kvx += ((invb - R(1)) * dxx - invb * V0) / rho;
          kvz += ((invb - R(1)) * dxz - invb * V1) / rho;
        }
        if (bottom) {
          const R dpb = dpz[iz] / bez[iz], apdpb = alz[iz] + dpb, invb = R(1) / bez[iz];
          const R V0 = S[SZVX][i], V1 = S[SZVZ][i];
          Kk[SZVX][i] = -apdpb * V0 + dpb * dzx;
          Kk[SZVZ][i] = -apdpb * V1 + dpb * dzz;
          kvx += ((invb - R(1)) * dzx - invb * V0) / rho;
          kvz += ((invb - R(1)) * dzz - invb * V1) / rho;
        }
        Kk[SVX][i] = kvx;
        Kk[SVZ][i] = kvz;
      }
    }
  }

  // 5x5 Gaussian point source added to the pressure RHS (include/tools_func.cuh:21-37).
  void add_source(R amp) {
    for (int j = -2; j <= 2; ++j)
      for (int i = -2; i <= 2; ++i) {
        const int ix = srcx + i, iz = srcz + j;
        if (ix <= 2 || ix >= nx - 3 || iz <= 2 || iz >= nzf - 3) continue;
        const R w = amp * R(kSrcW[j + 2][i + 2]);
        Kk[FP][size_t(iz) * nx + ix] += w;
      }
  }

  // Normal/tangential coupling of the interface-row RHS (include/pml_fs_kernels.cuh:754-827).
  void couple(int dir) {
    for (int ix = 3; ix <= nx - 4; ++ix) {
      const size_t f = size_t(nzf - 1) * nx + ix, s = ix;
      const R nxv = nfx[ix], nzv = nfz[ix];
      const R vxf = Kk[FVX][f], vzf = Kk[FVZ][f];
      R pf = Kk[FP][f];
      const R vxs = Kk[SVX][s], vzs = Kk[SVZ][s];
      const R sxx = Kk[SSX][s], szz = Kk[SSZ][s], sxz = Kk[SSXZ][s];
      R vnf = nxv * vxf + nzv * vzf;
      const R vtf = nzv * vxf - nxv * vzf;
      R vns = nxv * vxs + nzv * vzs;
      const R vts = nzv * vxs - nxv * vzs;
      R snn = nxv * nxv * sxx + 2 * nxv * nzv * sxz + nzv * nzv * szz;
      R snt = nxv * nzv * (sxx - szz) + (nzv * nzv - nxv * nxv) * sxz;
      const R stt = nzv * nzv * sxx - 2 * nxv * nzv * sxz + nxv * nxv * szz;
      if (dir == kF) { vnf = vns; pf = -snn; snt = 0; }
      else { vns = vnf; snn = -pf; snt = 0; }
      Kk[FVX][f] = nxv * vnf + nzv * vtf;
      Kk[FVZ][f] = nzv * vnf - nxv * vtf;
      Kk[FP][f] = pf;
      Kk[SVX][s] = nxv * vns + nzv * vts;
      Kk[SVZ][s] = nzv * vns - nxv * vts;
      Kk[SSX][s] = nxv * nxv * snn + 2 * nxv * nzv * snt + nzv * nzv * stt;
      Kk[SSZ][s] = nzv * nzv * snn - 2 * nxv * nzv * snt + nxv * nxv * stt;
      Kk[SSXZ][s] = -nxv * nzv * stt + (nzv * nzv - nxv * nxv) * snt;
    }
  }

  // Post-step interface filter and continuity average (src/pml_fs_kernels.cu:428-525),
  // evaluated out of place.
  void filter() {
    const size_t rf_ = size_t(nzf - 1) * nx;
    const R* src[8] = {&U[FVX][rf_], &U[FVZ][rf_], &U[FP][rf_], &U[SVX][0],
                       &U[SVZ][0],   &U[SSX][0],   &U[SSZ][0], &U[SSXZ][0]};
    std::vector<R> in(size_t(8) * nx);
    for (int f = 0; f < 8; ++f) std::memcpy(&in[size_t(f) * nx], src[f], sizeof(R) * nx);
    for (int ix = 3; ix <= nx - 4; ++ix) {
      const int klo = std::max(-3, 3 - ix), khi = std::min(3, nx - 4 - ix);
      R wsum = 0;
      for (int k = klo; k <= khi; ++k) wsum += R(kW7[k + 3]);
      R v[8];
      for (int f = 0; f < 8; ++f) {
        R sum = 0;
        for (int k = klo; k <= khi; ++k) sum += R(kW7[k + 3]) * in[size_t(f) * nx + ix + k];
        v[f] = sum / wsum;
      }
      const R nxv = nfx[ix], nzv = nfz[ix];
      const R vnf = nxv * v[0] + nzv * v[1], vtf = nzv * v[0] - nxv * v[1];
      const R vns = nxv * v[3] + nzv * v[4], vts = nzv * v[3] - nxv * v[4];
      const R snn = nxv * nxv * v[5] + R(2.0f) * nxv * nzv * v[7] + nzv * nzv * v[6];
      const R stt = nzv * nzv * v[5] - R(2.0f) * nxv * nzv * v[7] + nxv * nxv * v[6];
      const R vn = R(0.5f) * (vnf + vns);
      const R sn = R(0.5f) * (snn - v[2]);
      U[FVX][rf_ + ix] = nxv * vn + nzv * vtf;
      U[FVZ][rf_ + ix] = nzv * vn - nxv * vtf;
      U[FP][rf_ + ix] = -sn;
      U[SVX][ix] = nxv * vn + nzv * vts;
      U[SVZ][ix] = nzv * vn - nxv * vts;
      U[SSX][ix] = nxv * nxv * sn + nzv * nzv * stt;
      U[SSZ][ix] = nzv * nzv * sn + nxv * nxv * stt;
      U[SSXZ][ix] = nxv * nzv * (sn - stt);
    }
  }

  // Cells that can hold non-zero values: every cell of the state fields, and only
  // the strip cells of the ADE fields (elsewhere their RHS, and so their value, is 0).
  struct Job { int f, row, c0, c1, c2, c3; };  // columns [c0, c1) and [c2, c3)
  std::vector<Job> jobs;
  void build_jobs() {
    jobs.clear();
    for (int f = 0; f < NFIELD; ++f) {
      const int rows = is_fluid(f) ? nzf : nzs;
      const bool xstrip = (f >= FXVX && f <= SXEZ), zstrip = (f >= SZVX && f <= SZEZ);
      const bool fzstrip = f >= FZVX;
      for (int r = 0; r < rows; ++r) {
        if (zstrip && r < nzs - 3 - npd) continue;
        if (fzstrip && (!cpml || r < 3 || r > npd + 2)) continue;
        if (xstrip) jobs.push_back({f, r, 3, std::min(nx, 3 + npd), std::max(0, nx - 3 - npd), nx - 3});
        else jobs.push_back({f, r, 0, nx, 0, 0});
      }
    }
  }
  // Applies fn(field, flat index) to every live cell (OpenMP over rows).
  template <class Fn> void for_cells(Fn fn) {
#pragma omp parallel for schedule(static)
    for (long long j = 0; j < (long long)jobs.size(); ++j) {
      const Job& jb = jobs[size_t(j)];
      const size_t base = size_t(jb.row) * nx;
      for (int c = jb.c0; c < jb.c1; ++c) fn(jb.f, base + c);
      for (int c = jb.c2; c < jb.c3; ++c) fn(jb.f, base + c);
    }
  }

  // Stage input `S`: the state itself for the first stage, U_tmp afterwards.
  bool src_on = true;  // false: the stage RHS without the source (the linear operator alone)
  void stage(int dir, R t, const Set& S) {
    build_ghosts(S);
    fluid_velocity(dir, S);
    fluid_stress(dir, S);
    solid_velocity(dir, S);
    solid_stress(dir, S);
    if (src_on) add_source(ricker(t));
    couple(dir);
  }

  // Flat packing of a set: the NFIELD arrays [rows][nx] one after another.
  size_t set_len() const {
    size_t n = 0;
    for (int f = 0; f < NFIELD; ++f) n += size_t(is_fluid(f) ? nzf : nzs) * nx;
    return n;
  }
  void pack(const Set& S, double* out) const {
    for (int f = 0; f < NFIELD; ++f)
      for (size_t k = 0; k < S[f].size(); ++k) *out++ = double(S[f][k]);
  }
  void unpack(const double* in, Set& S) const {
    for (int f = 0; f < NFIELD; ++f)
      for (size_t k = 0; k < S[f].size(); ++k) S[f][k] = R(*in++);
  }

  // One RK4 step with direction order FBFB (even it) or BFBF (odd it)
  // (src/pml_fs_kernels.cu:765-868; src/main.cu:137-138). The reference first
  // copies U into U_b and U_tmp (src/elements.cu:345-383) and then applies
  // C = 1*A + c*B (matrix_add) and A += c*B (matrix_self_add,
  // src/common_kernels.cu:4-31); the same per-value arithmetic is applied here
  // without the copies: U_b = U + w1 k1 is exactly U_b += w1 k1 on a copy.
  // `save` (optional): the four stage inputs U, U_tmp, U_tmp, U_tmp, packed.
  void step(int it, double* save = nullptr) {
    const size_t sl = save ? set_len() : 0;
    if (save) pack(U, save);
    const int d0 = (it & 1) ? kB : kF, d1 = 1 - d0;
    R time, half, dt;
    if constexpr (std::is_same<R, float>::value) {
      time = R(float(it) * dt_f);
      half = R(float(double(dt_f) * 0.5));
      dt = R(dt_f);
    } else {
      time = R(double(it) * double(dt_f));
      half = R(0.5 * double(dt_f));
      dt = R(dt_f);
    }
    const R c_half = dt / 2, c_full = dt, w6 = dt / 6, w3 = dt / 3, w_last = dt / R(6.0f);
    stage(d0, time, U);
    for_cells([&](int f, size_t k) {
      Ut[f][k] = R(1) * U[f][k] + c_half * Kk[f][k];
      Ub[f][k] = U[f][k] + w6 * Kk[f][k];
    });
    if (save) pack(Ut, save + sl);
    stage(d1, time + half, Ut);
    for_cells([&](int f, size_t k) {
      Ut[f][k] = R(1) * U[f][k] + c_half * Kk[f][k];
      Ub[f][k] += w3 * Kk[f][k];
    });
    if (save) pack(Ut, save + 2 * sl);
    stage(d0, time + half, Ut);
    for_cells([&](int f, size_t k) {
      Ut[f][k] = R(1) * U[f][k] + c_full * Kk[f][k];
      Ub[f][k] += w3 * Kk[f][k];
    });
    if (save) pack(Ut, save + 3 * sl);
    stage(d1, time + dt, Ut);
    for_cells([&](int f, size_t k) { U[f][k] = R(1) * Ub[f][k] + w_last * Kk[f][k]; });
    filter();
  }
};

// ---- solid only with a free surface on top (PmlFs::SolidOnly) ----------------
// include/pml_fs_kernels.cuh:8-307, src/pml_fs_kernels.cu:5-381,
// src/elements.cu:824-873 (PML tables), 907-977 (ALM free-surface coefficients),
// src/main.cu:252-300 (the record: solid vz on row 3).
// The model's solid arrays and the metric are all [nz][nx] (nz = nz_s, nz_f
// unused): the solid fills the grid, the free surface is row 3, CFS-PML on the
// left, right and bottom.
// With m.cpml = 1 the same structure restates Cpml::SolidOnly
// (include/cpml_kernels.cuh:8-233, src/cpml_kernels.cu:5-361): CFS-PML on all
// four sides, no free surface - every row 3..nz-4 takes the plain biased
// operators (rows 0..2 read as zeros), the zeta-PML tables have a top band
// (rows 3..npd+2, src/elements.cu:869-871) whose cells share the zeta-ADE
// memory with the bottom band, and the record is solid vz on row 30
// (src/main.cu:303-311).
enum SField { TVX, TVZ, TSX, TSZ, TSXZ, XVX, XVZ, XEX, XEZ, ZVX, ZVZ, ZEX, ZEZ, NSFIELD };

template <class R>
struct SolidOracle {
  int nx, nz, npd;
  bool cpml;
  int rec_row;
  float fpeak_f, dt_f;
  int srcx, srcz;
  std::vector<R> C11, C13, C33, C55, rho, J, xx, xz, zx, zz;
  std::vector<R> alx, bex, dpx, alz, bez, dpz;
  std::vector<R> alm;  // [nx][6]: al1_xx, al1_zz, al1_xz, al2_xx, al2_zz, al2_xz
  using Set = std::vector<std::vector<R>>;
  Set U, Ub, Ut, Kk;

  static std::vector<R> conv(const double* p, size_t n) {
    std::vector<R> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = R(p[i]);
    return v;
  }
  void alloc(Set& S) { S.assign(NSFIELD, std::vector<R>(size_t(nz) * nx, R(0))); }

  explicit SolidOracle(const orc_model& m) {
    nx = m.nx; nz = m.nz_s; npd = m.npd;
    cpml = m.cpml != 0;
    rec_row = cpml ? 30 : 3;
    fpeak_f = float(m.fpeak); dt_f = float(m.dt);
    srcx = m.src_x; srcz = m.src_z;
    const size_t n = size_t(nz) * nx;
    C11 = conv(m.C11, n); C13 = conv(m.C13, n); C33 = conv(m.C33, n); C55 = conv(m.C55, n);
    rho = conv(m.rho_s, n);
    J = conv(m.J, n); xx = conv(m.xi_x, n); xz = conv(m.xi_z, n);
    zx = conv(m.ze_x, n); zz = conv(m.ze_z, n);
    alx.assign(nx, 0); bex.assign(nx, 0); dpx.assign(nx, 0);
    alz.assign(nz, 0); bez.assign(nz, 0); dpz.assign(nz, 0);
    pml_profile(m, fpeak_f, npd, alx.data(), bex.data(), dpx.data(), nx, true, true);
    pml_profile(m, fpeak_f, npd, alz.data(), bez.data(), dpz.data(), nz, cpml, true);
    if (!cpml) free_surface(m);
    alloc(U); alloc(Ub); alloc(Ut); alloc(Kk);
  }

  // ALM coefficients of the free-surface row (src/elements.cu:907-977): from
  // the traction-free condition the zeta derivatives of the velocity on row 3
  // are eliminated in favour of the xi derivatives; evaluated in double from
  // the model's float values (the FP64 oracle from its own values) and stored
  // at the oracle's precision.
  void free_surface(const orc_model& m) {
    alm.assign(size_t(nx) * 6, R(0));
    for (int ix = 0; ix < nx; ++ix) {
      const size_t i = size_t(3) * nx + ix;
      auto val = [&](const double* a) {
        return std::is_same<R, float>::value ? double(float(a[i])) : a[i];
      };
      const double xi_x = val(m.xi_x), xi_z = val(m.xi_z), ze_x = val(m.ze_x), ze_z = val(m.ze_z);
      const double c11 = val(m.C11), c13 = val(m.C13), c33 = val(m.C33), c55 = val(m.C55);
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
      R* a = &alm[size_t(ix) * 6];
      a[0] = R(xi_x - ze_x * m11);
      a[1] = R(-ze_z * m21);
      a[2] = R(xi_z - ze_z * m11 - ze_x * m21);
      a[3] = R(-ze_x * m12);
      a[4] = R(xi_z - ze_z * m22);
      a[5] = R(xi_x - ze_z * m12 - ze_x * m22);
    }
  }

  R ricker(R time) const {
    if constexpr (std::is_same<R, float>::value) {
      const float T = float(1.2 / double(fpeak_f));
      float t = float(time) - T;
      if (t > T) return 0.0f;
      float temp = float(M_PI * double(fpeak_f) * double(t));
      temp *= temp;
      return (1 - 2 * temp) * std::exp(-temp);
    }
    const double T = 1.2 / double(fpeak_f);
    double t = double(time) - T;
    if (t > T) return 0.0;
    double temp = M_PI * double(fpeak_f) * t;
    temp *= temp;
    return R((1 - 2 * temp) * std::exp(-temp));
  }

  // Solid flux rows (src/tools_func.cu:19-65 with no fluid above: no row offset).
  P2<R> flux_ze(const Set& S, int r, int ix) const {
    const size_t i = size_t(r) * nx + ix;
    return {J[i] * (zx[i] * S[TSX][i] + zz[i] * S[TSXZ][i]),
            J[i] * (zx[i] * S[TSXZ][i] + zz[i] * S[TSZ][i])};
  }
  P2<R> flux_xi(const Set& S, size_t i) const {
    return {J[i] * (xx[i] * S[TSX][i] + xz[i] * S[TSXZ][i]),
            J[i] * (xx[i] * S[TSXZ][i] + xz[i] * S[TSZ][i])};
  }

  // A cell of the zeta-PML band(s): the bottom band, and with cpml the top band.
  bool zeta_band(int iz) const { return iz >= nz - 3 - npd || (cpml && iz <= npd + 2); }

  void stress(int dir, const Set& S) {
#pragma omp parallel for schedule(static)
    for (int iz = 3; iz <= nz - 4; ++iz)
      for (int ix = 3; ix <= nx - 4; ++ix) {
        const size_t i = size_t(iz) * nx + ix;
        const int dist = cpml ? 3 : iz - 3, distx = std::min(ix - 3, nx - 4 - ix);
        const R dvx_dxi = dmac(dir, &S[TVX][i], 1), dvz_dxi = dmac(dir, &S[TVZ][i], 1);
        const bool side = distx < npd, bottom = zeta_band(iz);
        const R c11 = C11[i], c13 = C13[i], c33 = C33[i], c55 = C55[i];
        if (dist == 0) {
          const R* a = &alm[size_t(ix) * 6];
          Kk[TSX][i] = (c11 * a[0] + c13 * a[1]) * dvx_dxi + (c11 * a[3] + c13 * a[4]) * dvz_dxi;
          Kk[TSZ][i] = (c13 * a[0] + c33 * a[1]) * dvx_dxi + (c13 * a[3] + c33 * a[4]) * dvz_dxi;
          Kk[TSXZ][i] = c55 * (a[2] * dvx_dxi + a[5] * dvz_dxi);
          if (side) {
            const R dpb = dpx[ix] / bex[ix], apdpb = alx[ix] + dpb, invb = R(1) / bex[ix];
            const R E0 = S[XEX][i], E1 = S[XEZ][i];
            Kk[XEX][i] = -apdpb * E0 + dpb * dvx_dxi;
            Kk[XEZ][i] = -apdpb * E1 + dpb * dvz_dxi;
            const R cxx_x = c11 * a[0] + c13 * a[1], cxx_z = c11 * a[3] + c13 * a[4];
            Kk[TSX][i] += (invb - R(1)) * (cxx_x * dvx_dxi + cxx_z * dvz_dxi) -
                          invb * (cxx_x * E0 + cxx_z * E1);
            const R czz_x = c13 * a[0] + c33 * a[1], czz_z = c13 * a[3] + c33 * a[4];
            Kk[TSZ][i] += (invb - R(1)) * (czz_x * dvx_dxi + czz_z * dvz_dxi) -
                          invb * (czz_x * E0 + czz_z * E1);
            Kk[TSXZ][i] += c55 * ((invb - R(1)) * (a[2] * dvx_dxi + a[5] * dvz_dxi) -
                                  invb * (a[2] * E0 + a[5] * E1));
          }
          continue;
        }
        const R dvx_dze = dz_near(dir, &S[TVX][i], nx, dist, true);
        const R dvz_dze = dz_near(dir, &S[TVZ][i], nx, dist, true);
        const R xix = xx[i], xiz = xz[i], zex = zx[i], zez = zz[i];
        Kk[TSX][i] = c11 * (xix * dvx_dxi + zex * dvx_dze) + c13 * (xiz * dvz_dxi + zez * dvz_dze);
        Kk[TSZ][i] = c13 * (xix * dvx_dxi + zex * dvx_dze) + c33 * (xiz * dvz_dxi + zez * dvz_dze);
        Kk[TSXZ][i] = c55 * (xiz * dvx_dxi + zez * dvx_dze + xix * dvz_dxi + zex * dvz_dze);
        if (!side && !bottom) continue;
        const R gxixi = xix * xix + xiz * xiz, gxize = xix * zex + xiz * zez,
                gzeze = zex * zex + zez * zez;
        if (side) {
          const R Dvx = dvx_dxi + (gxize / gxixi) * dvx_dze, Dvz = dvz_dxi + (gxize / gxixi) * dvz_dze;
          const R dpb = dpx[ix] / bex[ix], apdpb = alx[ix] + dpb, invb = R(1) / bex[ix];
          const R E0 = S[XEX][i], E1 = S[XEZ][i];
          Kk[XEX][i] = -apdpb * E0 + dpb * Dvx;
          Kk[XEZ][i] = -apdpb * E1 + dpb * Dvz;
          Kk[TSX][i] += c11 * (invb - R(1)) * xix * Dvx + c13 * (invb - R(1)) * xiz * Dvz -
                        invb * c11 * xix * E0 - invb * c13 * xiz * E1;
          Kk[TSZ][i] += c13 * (invb - R(1)) * xix * Dvx + c33 * (invb - R(1)) * xiz * Dvz -
                        invb * c13 * xix * E0 - invb * c33 * xiz * E1;
          Kk[TSXZ][i] += c55 * (invb - R(1)) * (xiz * Dvx + xix * Dvz) - invb * c55 * xiz * E0 -
                         invb * c55 * xix * E1;
        }
        if (bottom) {
          const R Dvx = dvx_dze + (gxize / gzeze) * dvx_dxi, Dvz = dvz_dze + (gxize / gzeze) * dvz_dxi;
          const R dpb = dpz[iz] / bez[iz], apdpb = alz[iz] + dpb, invb = R(1) / bez[iz];
          const R E0 = S[ZEX][i], E1 = S[ZEZ][i];
          Kk[ZEX][i] = -apdpb * E0 + dpb * Dvx;
          Kk[ZEZ][i] = -apdpb * E1 + dpb * Dvz;
          Kk[TSX][i] += c11 * (invb - R(1)) * zex * Dvx + c13 * (invb - R(1)) * zez * Dvz -
                        invb * c11 * zex * E0 - invb * c13 * zez * E1;
          Kk[TSZ][i] += c13 * (invb - R(1)) * zex * Dvx + c33 * (invb - R(1)) * zez * Dvz -
                        invb * c13 * zex * E0 - invb * c33 * zez * E1;
          Kk[TSXZ][i] += c55 * (invb - R(1)) * (zez * Dvx + zex * Dvz) - invb * c55 * zez * E0 -
                         invb * c55 * zex * E1;
        }
      }
  }

  void velocity(int dir, const Set& S) {
#pragma omp parallel for schedule(static)
    for (int iz = 3; iz <= nz - 4; ++iz)
      for (int ix = 3; ix <= nx - 4; ++ix) {
        const size_t i = size_t(iz) * nx + ix;
        const int dist = cpml ? 3 : iz - 3;
        const R xix = xx[i], xiz = xz[i], zex = zx[i], zez = zz[i];
        const R gxixi = xix * xix + xiz * xiz, gzeze = zex * zex + zez * zez;
        R rvx, rvz, dxx, dxz, dzx, dzz;
        if (dist < 3) {
          // conservative rows below the free surface; above it the image G = -F
          // of the rows below (src/pml_fs_kernels.cu:7-19)
          auto Fxi = [&](int j) { return flux_xi(S, i + j); };
          auto Fze = [&](int j) -> P2<R> {
            const int r = iz + j;
            if (r >= 3) return flux_ze(S, r, ix);
            const P2<R> b = flux_ze(S, 6 - r, ix);
            return {-b.x, -b.y};
          };
          const P2<R> a = dflux<R>(dir, Fxi), b = dflux<R>(dir, Fze);
          rvx = (a.x + b.x) / J[i];
          rvz = (a.y + b.y) / J[i];
          const R gxize = xix * zex + xiz * zez;
          const R dxsx = dmac(dir, &S[TSX][i], 1), dxsz = dmac(dir, &S[TSZ][i], 1),
                  dxsxz = dmac(dir, &S[TSXZ][i], 1);
          const R dzsx = dz_near(dir, &S[TSX][i], nx, dist, true),
                  dzsz = dz_near(dir, &S[TSZ][i], nx, dist, true),
                  dzsxz = dz_near(dir, &S[TSXZ][i], nx, dist, true);
          dxx = xix * (dxsx + gxize / gxixi * dzsx) + xiz * (dxsxz + gxize / gxixi * dzsxz);
          dxz = xix * (dxsxz + gxize / gxixi * dzsxz) + xiz * (dxsz + gxize / gxixi * dzsz);
          dzx = 0;
          dzz = 0;
        } else {
          const R sxdx = dmac(dir, &S[TSX][i], 1), sxdz = dmac(dir, &S[TSX][i], nx);
          const R szdx = dmac(dir, &S[TSZ][i], 1), szdz = dmac(dir, &S[TSZ][i], nx);
          const R tdx = dmac(dir, &S[TSXZ][i], 1), tdz = dmac(dir, &S[TSXZ][i], nx);
          rvx = xix * sxdx + zex * sxdz + xiz * tdx + zez * tdz;
          rvz = xix * tdx + zex * tdz + xiz * szdx + zez * szdz;
          const R gxize = xix * zex + xiz * zez;
          dxx = xix * (sxdx + gxize / gxixi * sxdz) + xiz * (tdx + gxize / gxixi * tdz);
          dxz = xix * (tdx + gxize / gxixi * tdz) + xiz * (szdx + gxize / gxixi * szdz);
          dzx = zex * (sxdz + gxize / gzeze * sxdx) + zez * (gxize / gzeze * tdx + tdz);
          dzz = zex * (gxize / gzeze * tdx + tdz) + zez * (gxize / gzeze * szdx + szdz);
        }
        const int distx = std::min(ix - 3, nx - 4 - ix);
        const bool side = distx < npd, bottom = zeta_band(iz);
        const R r0 = rho[i];
        R kvx = rvx / r0, kvz = rvz / r0;
        if (side) {
          const R dpb = dpx[ix] / bex[ix], apdpb = alx[ix] + dpb, invb = R(1) / bex[ix];
          const R V0 = S[XVX][i], V1 = S[XVZ][i];
          Kk[XVX][i] = -apdpb * V0 + dpb * dxx;
          Kk[XVZ][i] = -apdpb * V1 + dpb * dxz;
          kvx += ((invb - R(1)) * dxx - invb * V0) / r0;
          kvz += ((invb - R(1)) * dxz - invb * V1) / r0;
        }
        if (bottom) {
          const R dpb = dpz[iz] / bez[iz], apdpb = alz[iz] + dpb, invb = R(1) / bez[iz];
          const R V0 = S[ZVX][i], V1 = S[ZVZ][i];
          Kk[ZVX][i] = -apdpb * V0 + dpb * dzx;
          Kk[ZVZ][i] = -apdpb * V1 + dpb * dzz;
          kvx += ((invb - R(1)) * dzx - invb * V0) / r0;
          kvz += ((invb - R(1)) * dzz - invb * V1) / r0;
        }
        Kk[TVX][i] = kvx;
        Kk[TVZ][i] = kvz;
      }
  }

  // Explosive source: the 5x5 Gaussian added to both normal stresses
  // (src/pml_fs_kernels.cu:22-26, include/tools_func.cuh:21-37).
  void add_source(R amp) {
    for (int j = -2; j <= 2; ++j)
      for (int q = -2; q <= 2; ++q) {
        const int ix = srcx + q, iz = srcz + j;
        if (ix <= 2 || ix >= nx - 3 || iz <= 2 || iz >= nz - 3) continue;
        const R w = amp * R(kSrcW[j + 2][q + 2]);
        const size_t i = size_t(iz) * nx + ix;
        Kk[TSX][i] += w;
        Kk[TSZ][i] += w;
      }
  }

  void stage(int dir, R t, const Set& S) {
    velocity(dir, S);
    stress(dir, S);
    add_source(ricker(t));
  }

  // Live cells: every cell of the five state fields, the strip cells of the ADE fields.
  bool live(int f, int iz, int ix) const {
    if (f < XVX) return true;
    if (f < ZVX) {
      const int d = std::min(ix - 3, nx - 4 - ix);
      return ix >= 3 && ix <= nx - 4 && d < npd;
    }
    return iz >= 3 && iz <= nz - 4 && zeta_band(iz);
  }
  template <class Fn> void for_cells(Fn fn) {
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nz; ++iz)
      for (int f = 0; f < NSFIELD; ++f)
        for (int ix = 0; ix < nx; ++ix)
          if (live(f, iz, ix)) fn(f, size_t(iz) * nx + ix);
  }

  // One RK4 step (src/pml_fs_kernels.cu:95-380), the same stage weights and
  // direction order as the fluid-solid step.
  void step(int it) {
    const int d0 = (it & 1) ? kB : kF, d1 = 1 - d0;
    R time, half, dt;
    if constexpr (std::is_same<R, float>::value) {
      time = R(float(it) * dt_f);
      half = R(float(double(dt_f) * 0.5));
      dt = R(dt_f);
    } else {
      time = R(double(it) * double(dt_f));
      half = R(0.5 * double(dt_f));
      dt = R(dt_f);
    }
    const R c_half = dt / 2, c_full = dt, w6 = dt / 6, w3 = dt / 3, w_last = dt / R(6.0f);
    stage(d0, time, U);
    for_cells([&](int f, size_t k) {
      Ut[f][k] = R(1) * U[f][k] + c_half * Kk[f][k];
      Ub[f][k] = U[f][k] + w6 * Kk[f][k];
    });
    stage(d1, time + half, Ut);
    for_cells([&](int f, size_t k) {
      Ut[f][k] = R(1) * U[f][k] + c_half * Kk[f][k];
      Ub[f][k] += w3 * Kk[f][k];
    });
    stage(d0, time + half, Ut);
    for_cells([&](int f, size_t k) {
      Ut[f][k] = R(1) * U[f][k] + c_full * Kk[f][k];
      Ub[f][k] += w3 * Kk[f][k];
    });
    stage(d1, time + dt, Ut);
    for_cells([&](int f, size_t k) { U[f][k] = R(1) * Ub[f][k] + w_last * Kk[f][k]; });
  }
};

template <class R>
int run_solid(const orc_model* m, int nsteps, int gap, double* rvz, double* out) {
  SolidOracle<R> o(*m);
  const int nx = m->nx;
  for (int it = 0; it < nsteps; ++it) {
    o.step(it);
    if (gap > 0 && it % gap == 0 && rvz)
      for (int ix = 0; ix < nx; ++ix)
        rvz[size_t(it / gap) * nx + ix] = double(o.U[TVZ][size_t(o.rec_row) * nx + ix]);
  }
  if (out) {
    const size_t n = size_t(m->nz_s) * nx;
    for (int q = 0; q < 5; ++q)
      for (size_t k = 0; k < n; ++k) out[q * n + k] = double(o.U[q][k]);
  }
  return 0;
}

template <class R>
int run(const orc_model* m, int nsteps, int gap, double* rvx, double* rvz, double* rp,
        double* out_fluid, double* out_solid) {
  Oracle<R> o(*m);
  const int nx = m->nx;
  for (int it = 0; it < nsteps; ++it) {
    o.step(it);
    if (gap > 0 && it % gap == 0) {
      const size_t s = size_t(it / gap) * nx;
      const size_t rf_ = size_t(m->nz_f - 1) * nx;
      for (int ix = 0; ix < nx; ++ix) {
        if (rvx) rvx[s + ix] = double(o.U[SVX][ix]);
        if (rvz) rvz[s + ix] = double(o.U[SVZ][ix]);
        if (rp) rp[s + ix] = double(o.U[FP][rf_ + ix]);
      }
    }
  }
  if (out_fluid) {
    const size_t n = size_t(m->nz_f) * nx;
    const int ff[3] = {FVX, FVZ, FP};
    for (int q = 0; q < 3; ++q)
      for (size_t k = 0; k < n; ++k) out_fluid[q * n + k] = double(o.U[ff[q]][k]);
  }
  if (out_solid) {
    const size_t n = size_t(m->nz_s) * nx;
    const int fs[5] = {SVX, SVZ, SSX, SSZ, SSXZ};
    for (int q = 0; q < 5; ++q)
      for (size_t k = 0; k < n; ++k) out_solid[q * n + k] = double(o.U[fs[q]][k]);
  }
  return 0;
}

}  // namespace

extern "C" {

// Runs `nsteps` RK4 steps from a zero wavefield (shot 0) and returns the
// interface records every `gap` steps and, optionally, the final fields.
// precision: 32 or 64. nthreads <= 0 keeps the OpenMP default.
// Record arrays are [ceil(nsteps/gap)][nx]; out_fluid is [3][nz_f][nx]
// (vx, vz, p); out_solid is [5][nz_s][nx] (vx, vz, sx, sz, sxz).
int orc_forward(const orc_model* m, int precision, int nsteps, int gap, double* rec_svx,
                double* rec_svz, double* rec_fp, double* out_fluid, double* out_solid,
                int nthreads) {
  if (!m || m->nx < 8 || m->nz_f < 8 || m->nz_s < 8 || nsteps < 0) return -1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  // Far from the wavefront the stencil spreads values that decay into the
  // subnormal range, where x86 arithmetic is about 100x slower. Flush them to
  // zero for the duration of the call (FTZ + DAZ on every OpenMP thread, the
  // previous MXCSR restored afterwards); values below 1.2e-38 do not change
  // any record at the 1e-5 level the oracle is used for.
  unsigned saved = _mm_getcsr();
#pragma omp parallel
  { _mm_setcsr(_mm_getcsr() | 0x8040u); }
  _mm_setcsr(saved | 0x8040u);
  const int rc = precision == 64
                     ? run<double>(m, nsteps, gap, rec_svx, rec_svz, rec_fp, out_fluid, out_solid)
                     : run<float>(m, nsteps, gap, rec_svx, rec_svz, rec_fp, out_fluid, out_solid);
#pragma omp parallel
  { _mm_setcsr(saved); }
  _mm_setcsr(saved);
  return rc;
}

// Solid only with a free surface (PmlFs::SolidOnly), or with CFS-PML on all four
// sides (Cpml::SolidOnly) when m->cpml: nz_s is the grid's row count, the solid
// and metric arrays are [nz_s][nx], nz_f and the fluid arrays are unused.
// Records: solid vz on row 3 (row 30 with cpml) every `gap` steps ([ceil(nsteps/gap)][nx]);
// out_solid: the final [5][nz_s][nx] (vx, vz, sx, sz, sxz).
int orc_forward_solid(const orc_model* m, int precision, int nsteps, int gap, double* rec_vz,
                      double* out_solid, int nthreads) {
  if (!m || m->nx < 8 || m->nz_s < 8 || nsteps < 0) return -1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  unsigned saved = _mm_getcsr();
#pragma omp parallel
  { _mm_setcsr(_mm_getcsr() | 0x8040u); }
  _mm_setcsr(saved | 0x8040u);
  const int rc = precision == 64 ? run_solid<double>(m, nsteps, gap, rec_vz, out_solid)
                                 : run_solid<float>(m, nsteps, gap, rec_vz, out_solid);
#pragma omp parallel
  { _mm_setcsr(saved); }
  _mm_setcsr(saved);
  return rc;
}

// Persistent handle for timing: create once, advance in chunks, destroy.
struct orc_handle {
  int precision;
  void* impl;
  int it;
};

orc_handle* orc_create(const orc_model* m, int precision) {
  if (!m || m->nx < 8 || m->nz_f < 8 || m->nz_s < 8) return nullptr;
  orc_handle* h = new orc_handle{precision, nullptr, 0};
  if (precision == 64) h->impl = new Oracle<double>(*m);
  else h->impl = new Oracle<float>(*m);
  return h;
}

// Advances nsteps steps (same FTZ/DAZ handling as orc_forward); nthreads <= 0 keeps the default.
int orc_step(orc_handle* h, int nsteps, int nthreads) {
  if (!h || nsteps < 0) return -1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  unsigned saved = _mm_getcsr();
#pragma omp parallel
  { _mm_setcsr(_mm_getcsr() | 0x8040u); }
  _mm_setcsr(saved | 0x8040u);
  for (int k = 0; k < nsteps; ++k, ++h->it) {
    if (h->precision == 64) static_cast<Oracle<double>*>(h->impl)->step(h->it);
    else static_cast<Oracle<float>*>(h->impl)->step(h->it);
  }
#pragma omp parallel
  { _mm_setcsr(saved); }
  _mm_setcsr(saved);
  return 0;
}

void orc_destroy(orc_handle* h) {
  if (!h) return;
  if (h->precision == 64) delete static_cast<Oracle<double>*>(h->impl);
  else delete static_cast<Oracle<float>*>(h->impl);
  delete h;
}

// ---- linearised pieces for the FP64 adjoint oracle ----------------------------
// A set is packed as the NFIELD arrays in Field order, fluid-sized fields
// [nz_f][nx], solid-sized [nz_s][nx].

long long orc_set_len(orc_handle* h) {
  if (!h) return -1;
  return h->precision == 64 ? (long long)static_cast<Oracle<double>*>(h->impl)->set_len()
                            : (long long)static_cast<Oracle<float>*>(h->impl)->set_len();
}

extern "C++" template <class R>
int rhs_impl(Oracle<R>* o, int dir, const double* in, double* out) {
  typename Oracle<R>::Set S;
  o->alloc(S);
  o->unpack(in, S);
  for (auto& f : o->Kk) std::fill(f.begin(), f.end(), R(0));
  const bool src = o->src_on;
  o->src_on = false;
  o->stage(dir, R(0), S);
  o->src_on = src;
  o->pack(o->Kk, out);
  return 0;
}

// out = the stage right-hand side of the packed set `in` with operator
// direction `dir` (0 F, 1 B), without the source: the linear operator L_dir,
// interface coupling included.
int orc_rhs(orc_handle* h, int dir, const double* in, double* out) {
  if (!h || !in || !out || (dir != 0 && dir != 1)) return -1;
  return h->precision == 64 ? rhs_impl(static_cast<Oracle<double>*>(h->impl), dir, in, out)
                            : rhs_impl(static_cast<Oracle<float>*>(h->impl), dir, in, out);
}

extern "C++" template <class R>
int filter_impl(Oracle<R>* o, double* set) {
  typename Oracle<R>::Set keep = o->U;
  o->unpack(set, o->U);
  o->filter();
  o->pack(o->U, set);
  o->U = keep;
  return 0;
}

// Applies the post-step interface filter to the packed set in place.
int orc_filter(orc_handle* h, double* set) {
  if (!h || !set) return -1;
  return h->precision == 64 ? filter_impl(static_cast<Oracle<double>*>(h->impl), set)
                            : filter_impl(static_cast<Oracle<float>*>(h->impl), set);
}

// Reads / replaces the state (and sets the step index of the next step).
int orc_get_state(orc_handle* h, double* set) {
  if (!h || !set) return -1;
  if (h->precision == 64) { auto* o = static_cast<Oracle<double>*>(h->impl); o->pack(o->U, set); }
  else { auto* o = static_cast<Oracle<float>*>(h->impl); o->pack(o->U, set); }
  return 0;
}
int orc_set_state(orc_handle* h, const double* set, int it) {
  if (!h || !set || it < 0) return -1;
  if (h->precision == 64) { auto* o = static_cast<Oracle<double>*>(h->impl); o->unpack(set, o->U); }
  else { auto* o = static_cast<Oracle<float>*>(h->impl); o->unpack(set, o->U); }
  h->it = it;
  return 0;
}

// One step at the handle's step index, the four stage inputs packed into
// `save` (4 sets), then the index advances.
int orc_step_save(orc_handle* h, double* save) {
  if (!h || !save) return -1;
  unsigned saved = _mm_getcsr();
#pragma omp parallel
  { _mm_setcsr(_mm_getcsr() | 0x8040u); }
  _mm_setcsr(saved | 0x8040u);
  if (h->precision == 64) static_cast<Oracle<double>*>(h->impl)->step(h->it, save);
  else static_cast<Oracle<float>*>(h->impl)->step(h->it, save);
#pragma omp parallel
  { _mm_setcsr(saved); }
  _mm_setcsr(saved);
  ++h->it;
  return 0;
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
