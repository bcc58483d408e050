// Adjoint-state backward of the RK4 time step (library-internal).
//
// The reference has no adjoint. This is the exact discrete adjoint of the
// library's own forward step: every piece of the step is linear in the state,
// so its transpose is assembled or derived from the forward kernels rather than
// written out by hand for every boundary case.
//
// * The stage operators L_F and L_B (the stage right-hand side without the
//   source, interface coupling included) are assembled once per model as CSR
//   matrices of L^T by probing the forward stage kernel: every output of the
//   stencil depends on inputs at most 3 cells away in x and in the global row,
//   so one stage launch on an input field that is 1 on a 7 x 7 lattice and 0
//   elsewhere yields 1/49 of that field's columns, each output attributable to
//   exactly one input.
// * The interface filter's transpose and the RK4 bookkeeping are written out
//   (they are short); the coupling uses the same device functions as the
//   forward kernels.
// * The derivative of a stage RHS with respect to one material coefficient of
//   a cell is the RHS of that cell evaluated with the coefficient set to 1 and
//   the others to 0, the forward's own RHS functions with another coefficient
//   set.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "mfdm_device.cuh"

namespace mfdm {

constexpr int kSetArrays = 24;  // state arrays of one RK set (fluid, solid, ADE strips)

// Where every array of one RK set sits inside the set's contiguous range, and
// how its cells map to global (row, column): fluid rows are global rows,
// solid row r is global row nz_f - 1 + r, xi-strip slots are the columns
// 3..npd+2 and nx-3-npd..nx-4, the solid zeta strip starts at solid row
// nz_s - 3 - npd and the fluid top band at fluid row 3.
struct SetLayout {
  long long len;                    // floats per set
  long long off[kSetArrays];        // first float of each array
  int rows[kSetArrays];             // rows of each array (0: absent)
  int pitch[kSetArrays];            // floats per row
  int ncols[kSetArrays];            // valid columns per row
  int kind[kSetArrays];             // 0 fluid, 1 solid, 2 fluid xi strip, 3 solid xi strip,
                                    // 4 solid zeta strip, 5 fluid zeta band
  int nx, nzf, nzs, npd;
  int cpml;                         // four-side CFS-PML (fluid top band, no free surface)
};

// Transposed stage operator of one direction: row j of L^T (an input value of
// the stage) lists the outputs that read it.
struct CsrT {
  long long* rowptr = nullptr;  // len + 1
  int* col = nullptr;
  float* val = nullptr;
  long long nnz = 0;
};

// The transposed operator in two parts. Output cells where the forward stage
// takes the plain interior formula (no PML strip, no conservative or
// one-sided row, not the interface) contribute through the transposed stencil:
// there L = (material x metric) . D, and the biased DRP pair satisfies
// D_F^T = -D_B and D_B^T = -D_F, so L^T x is the opposite-bias derivative of the
// point-wise products of x with the cell's coefficients (the Q fields). All
// other outputs contribute through the CSR (the probed operator with the
// interior outputs dropped).
struct HybridT {
  CsrT rest;              // CSR of L^T restricted to non-interior outputs
  int* nzrow = nullptr;   // rows of `rest` that have entries
  long long nrows = 0;
  float* t = nullptr;     // set-sized: the CSR part of each row (0 on rows without entries)
  float* qx = nullptr;    // set-sized: xi-direction products, by input field
  float* qz = nullptr;    // set-sized: zeta-direction products
};

namespace adj {

// Sets `v` at the cells of array `a` on lattice point (cz, cx) (global row mod 7, column mod 7).
cudaError_t set_lattice(float* set, const SetLayout& L, int a, int cz, int cx, float v, cudaStream_t st);
// Fills the whole set with v.
cudaError_t fill(float* set, long long n, float v, cudaStream_t st);
// mask[i] = out[i] != 0.
cudaError_t make_mask(const float* out, uint8_t* mask, long long n, cudaStream_t st);
// Attributes every non-zero output of a lattice probe of array `a` to its
// input. Pass 1 (rowptr == nullptr): count[j]++; pass 2: writes col / val
// (value / scale) at rowptr[j] + cursor[j]++. Unattributable outputs raise *err.
cudaError_t extract(const float* out, const SetLayout& L, int a, int cz, int cx, float scale,
                    unsigned long long* count, const long long* rowptr, int* cursor, int* col,
                    float* val, int* err, cudaStream_t st);
// rowptr = exclusive prefix sum of count (len + 1 entries); scratch from *tmp.
cudaError_t scan(const unsigned long long* count, long long* rowptr, long long len, void** tmp,
                 size_t* tmp_bytes, cudaStream_t st);
// Sorts every row of the CSR by column (deterministic sums).
cudaError_t sort_rows(const CsrT& A, long long len, cudaStream_t st);

// Drops from `full` the entries whose output lies in the interior set, into
// `rest` (allocated here); count and tmp are scratch.
cudaError_t drop_interior(const CsrT& full, const SetLayout& L, CsrT* rest,
                          unsigned long long* count, void** tmp, size_t* tmp_bytes, cudaStream_t st);

// The Q fields of kb into H.qx / H.qz (the interior and strip cells; 0 off
// them) and its sparse rows of L^T kb into H.t (the rows listed in H.nzrow),
// in one launch.
cudaError_t prepare(const HybridT& H, const Coef& C, const SetLayout& L, const float* kb,
                    cudaStream_t st);
// One reverse stage: y = L^T kb, lam += (mask_lam ? M : 1) y and, when kbn is
// given, kbn = M (w mu + c y); without mask_lam (the step's last stage) and
// with kbn, it also starts the next transposed step: mu = lam, kbn = w M lam.
// q_ready: the Q fields of kb and its sparse rows (prepare()) are already in H. lam_from_mu (with mask_lam and kbn: the step's first
// stage) reads lam from mu, which holds the step start's filtered lam.
cudaError_t reverse_stage(const HybridT& H, const Coef& C, const SetLayout& L, int dir,
                          const float* kb, float* lam, const uint8_t* mask, bool mask_lam,
                          float* kbn, float* mu, float w, float c, bool q_ready, bool lam_from_mu,
                          cudaStream_t st);
// Lists the rows of H->rest that have entries and allocates H->t (zeroed);
// flag (len + 1) and tmp are scratch.
cudaError_t list_rows(HybridT* H, const SetLayout& L, unsigned long long* flag, void** tmp,
                      size_t* tmp_bytes, cudaStream_t st);
// x = uniform pseudo-random values in [-1, 1) (self-checks).
cudaError_t random_fill(float* x, long long n, unsigned seed, cudaStream_t st);
// y = L^T x through the hybrid (H) or through a plain CSR (H.qx == nullptr).
cudaError_t apply_t(const HybridT& H, const Coef& C, const SetLayout& L, int dir, const float* x,
                    float* y, cudaStream_t st);

// The start of one transposed step, in one launch: with res (the residuals of
// the step's receiver sample, svx, svz, fp rows of nx) added to lam's
// interface cells, the transposed post-step filter F^T lam of the interface
// columns goes to mu and kb = c M mu there (off those cells both were formed
// by the previous transposed step, with mu = lam). lam is only read: the step's
// first transposed stage takes lam from mu (reverse_stage, lam_from_mu).
cudaError_t step_start(const float* lam, const SetLayout& L, const Coef& C, const float* res,
                       float* mu, float* kb, const uint8_t* mask, float c, cudaStream_t st);

// Material gradients of one stage: g[m][cell] += kb . dL_dir/dm (Y) over the
// cell's main fields (and the coupled interface column); Y is a set, kb a
// set-sized buffer. g: K, 1/rho_f ([nz_f][P]) then C11, C13, C33, C55,
// 1/rho_s ([nz_s][P]). With H, the Q fields of kb for H's transposed operator
// are written on the way (the interior cells; the rest of H's Q buffers must
// hold 0).
cudaError_t gradient(const Coef& C, const SetLayout& L, const Fields& Y, const float* kb,
                     double* const* g, int dir, HybridT* H, cudaStream_t st);

}  // namespace adj
}  // namespace mfdm
