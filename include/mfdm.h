/*
 * mfdm.h - C ABI of the B200 fluid-solid time-stepping library (libmfdm.so).
 *
 * Drop-in replacement of MarineSeis-FDM-2D's time-stepping path for the
 * pressure-free-top configuration (calc_type 1 = FANDS, boundary_type 2 =
 * PANDF): a fluid layer over an elastic solid on a curvilinear grid, classical
 * RK4 with alternating DRP MacCormack-type operators, ADE CFS-PML on the left,
 * right and bottom, the free surface on row 3, seafloor coupling, a Ricker
 * point source and interface receivers. The reference exposes this path only
 * as a C++ function and a command line, so every entry point below cites the
 * reference code it replaces (paths inside the reference project).
 *
 * Conventions: every function returns MFDM_OK (0) or a negative MFDM_ERR_*
 * code and never exits the process; mfdm_last_error() returns the message of
 * the calling thread's last failure. Handles are opaque and must be used by
 * one host thread at a time. Host arrays are caller-owned, row-major
 * [rows][nx] float32; device memory is owned by the handle.
 */
#ifndef MFDM_H
#define MFDM_H

#ifdef __cplusplus
extern "C" {
#endif

#define MFDM_OK 0
#define MFDM_ERR_ARG (-1)         /* bad argument or unsupported configuration   */
#define MFDM_ERR_IO (-2)          /* file missing, short read, write failure     */
#define MFDM_ERR_CONFIG (-3)      /* JSON syntax, missing key or type mismatch   */
#define MFDM_ERR_CUDA (-4)        /* CUDA runtime error                          */
#define MFDM_ERR_NONFINITE (-5)   /* NaN/Inf reached the interface rows          */
#define MFDM_ERR_NOMEM (-6)       /* device allocation failed                    */

typedef struct mfdm_model mfdm_model;

/* In-memory model description; field meaning follows json_template.json:1-50
 * and src/elements.cu:72-154. nz_f and nz_s both include the interface row;
 * the metric arrays cover nz_f + nz_s - 1 global rows. */
typedef struct mfdm_desc {
  int nx, nz_f, nz_s;
  float fpeak, dt;
  int nt, snapshot;
  int npd, npow;
  float thickness, vp_max, rc, beta0;
  int nsrc;
  const int* src_x;               /* [nsrc] source columns            */
  const int* src_z;               /* [nsrc] source fluid rows         */
  const float* K;                 /* [nz_f][nx] fluid bulk modulus    */
  const float* rho_f;             /* [nz_f][nx] fluid density         */
  const float* C11;               /* [nz_s][nx] solid stiffness       */
  const float* C13;
  const float* C33;
  const float* C55;
  const float* rho_s;             /* [nz_s][nx] solid density         */
  const float* J;                 /* [nz_f+nz_s-1][nx] metric         */
  const float* xi_x;
  const float* xi_z;
  const float* ze_x;
  const float* ze_z;
  int boundary_type;              /* 2 (or 0): free surface on top, CFS-PML on the other
                                     sides; 1: CFS-PML on all four sides (the reference's
                                     grid.boundary_type, Cpml::FluidSolid)              */
} mfdm_desc;

typedef struct mfdm_info {
  int nx, nz_f, nz_s, pitch;
  int nt, snapshot, gap, nsrc, shot;
  int step;                       /* time index of the next step      */
  int nsamples;                   /* receiver samples recorded so far */
  long long cells;                /* nx * (nz_f + nz_s): cells updated per step */
  long long device_bytes;         /* device memory held by the handle */
  int nshots;                     /* shots stepped together (1 unless opened with mfdm_open_batch) */
  int seg_rows;                   /* rows per segment block of the stage launches */
  int blocks_per_sm;              /* stage kernel build in use: 2 or 3 (TMA rings), 4 (tiles) */
} mfdm_info;

/* Field ids for mfdm_get_field / mfdm_set_field. */
#define MFDM_FLUID_VX 0
#define MFDM_FLUID_VZ 1
#define MFDM_FLUID_P 2
#define MFDM_SOLID_VX 3
#define MFDM_SOLID_VZ 4
#define MFDM_SOLID_SX 5
#define MFDM_SOLID_SZ 6
#define MFDM_SOLID_SXZ 7

/* Thread-local message of the last failing call ("" if none). */
const char* mfdm_last_error(void);

/* Reads a JSON config and its .bin arrays and uploads them to `device`.
 * Replaces MemManager::MemManager(const char*) + grid_cp_h2d()
 * (src/elements.cu:64-183, 307-333); relative paths resolve against the
 * working directory as in the reference. */
int mfdm_open_json(const char* json_path, int device, mfdm_model** out);

/* Same from host arrays (no files); the arrays are copied. */
int mfdm_open_desc(const mfdm_desc* desc, int device, mfdm_model** out);

/* Re-uploads the model arrays and scalars of `desc` into an open handle with
 * the same nx, nz_f, nz_s and npd (a new model for the next shot or
 * iteration without reallocating). The wavefield is left untouched; call
 * mfdm_set_shot to restart. */
int mfdm_load_desc(mfdm_model* m, const mfdm_desc* desc);

/* Frees the handle and its device memory (MemManager::~MemManager, src/elements.cu:186-304). */
int mfdm_close(mfdm_model* m);

int mfdm_get_info(const mfdm_model* m, mfdm_info* info);

/* Selects shot `isrc` (source position), rewinds the time index to 0 and
 * clears the receiver buffer. reset_state = 1 also zeroes the wavefield and
 * ADE memory; 0 keeps them, which is what the reference's shot loop does
 * (src/main.cu:94-136 never clears the fields between shots). */
int mfdm_set_shot(mfdm_model* m, int isrc, int reset_state);

/* One RK4 step for time index `it` (direction order FBFB for even it, BFBF
 * for odd, src/main.cu:137-138) followed by the interface filter and the
 * receiver sample when it % gap == 0. Replaces PmlFs::FluidSolid::update_RK4
 * (include/pml_fs_kernels.cuh:848-852, src/pml_fs_kernels.cu:765-868) plus
 * MemManager::RK4_reset (src/elements.cu:345-383), which is fused away.
 * `stream` is a cudaStream_t (NULL = the handle's stream); asynchronous. */
int mfdm_update_rk4(mfdm_model* m, int it, void* stream);

/* Advances `nsteps` steps from the current time index on the handle's stream
 * through a captured CUDA graph (the time loop of src/main.cu:136-213 without
 * the host I/O), then synchronises and checks the non-finite flag. */
int mfdm_step(mfdm_model* m, int nsteps);

/* Advances `nsteps` steps like mfdm_step and reports device time measured
 * with CUDA events on the handle's stream: *total_ms for the whole run. With
 * per_kernel != 0 the steps are launched one by one (back to back, outside the
 * graph) with an event between consecutive kernels, and kernel_ms[0..3] receive
 * the summed time of the four RK stage launches and kernel_ms[4] that of the
 * filter/receiver launch. */
int mfdm_time_steps(mfdm_model* m, int nsteps, int per_kernel, float* total_ms, float* kernel_ms);

/* Waits for the handle's stream. */
int mfdm_synchronize(mfdm_model* m);

/* Copies receiver samples [first, first + count) to host arrays of
 * [count][nx] floats each (any may be NULL): solid vx and vz on solid row 0
 * and fluid pressure on fluid row nz_f - 1, the rows the reference appends to
 * record/solid_vx.bin, solid_vz.bin and fluid_p.bin (src/main.cu:245-295). */
int mfdm_get_records(mfdm_model* m, int first, int count, float* solid_vx, float* solid_vz,
                     float* fluid_p);

/* Copies one state field to/from a host array of [rows][nx] floats
 * (MemManager::U_cp_d2h, src/elements.cu:335-343, for the snapshot writer). */
int mfdm_get_field(mfdm_model* m, int field, float* host);
int mfdm_set_field(mfdm_model* m, int field, const float* host);

/* ---- batched shots ------------------------------------------------------
 * Several shots of one model stepped together: one launch per RK stage covers
 * every shot (the model's coefficients are shared, each shot has its own
 * wavefield). The reference runs shots one after another from one JSON
 * (src/main.cu:94-136) without clearing the wavefield between them and with
 * one frequency for all; here every shot starts from rest and carries its own
 * source cell and Ricker frequency, with the CFS-PML alpha0 = 2 pi fpeak and
 * beta0 that go with it (elements.cu:121-124, 824-873). */
typedef struct mfdm_shot {
  int src_x, src_z;  /* source column and fluid row (src_x < 0: no source) */
  float fpeak;       /* Ricker peak frequency, Hz                           */
  float beta0;       /* CFS-PML beta0 for this shot (>= 1)                  */
} mfdm_shot;

/* Opens `nshots` shots on the model of `d` (d->src_* and d->fpeak / d->beta0
 * are not used). mfdm_step / mfdm_time_steps / mfdm_synchronize / mfdm_close
 * act on all shots; mfdm_get_records / mfdm_get_field read shot 0;
 * mfdm_set_shot is rejected (MFDM_ERR_ARG). */
int mfdm_open_batch(const mfdm_desc* d, int nshots, const mfdm_shot* shots, int device,
                    mfdm_model** out);
/* Every shot back to rest, step counter to 0, records cleared. */
int mfdm_batch_reset(mfdm_model* m);
/* Receiver rows / state field of one shot (as mfdm_get_records / mfdm_get_field). */
int mfdm_batch_get_records(mfdm_model* m, int shot, int first, int count, float* svx, float* svz,
                           float* fp);
int mfdm_batch_get_field(mfdm_model* m, int shot, int field, float* host);

/* ---- tile shape ---------------------------------------------------------
 * A stage launch covers each medium with segment blocks of 64 columns by
 * `seg_rows` rows. Small grids want short segments (more blocks than SMs),
 * large ones long segments (fewer halo re-reads). The reference launches
 * fixed 16x16 blocks (src/pml_fs_kernels.cu:533-622) and has no tuner. */

/* Sets the segment height: a multiple of 4 in [4, 128], or 0 for the default
 * (24 from 6 M cells per launch, counting every shot of a batch, 8 below; the
 * tile build, mfdm_set_blocks_per_sm 4, rounds it up to a multiple of 8 and
 * caps it at 48, 16 by default). Results do not depend on it beyond FP32
 * rounding of the last bit. */
int mfdm_set_tile(mfdm_model* m, int seg_rows);

/* Selects the stage kernel build: 2 resident blocks per SM (deeper TMA rings,
 * 96 registers) or 3 (shallower rings, 72 registers, more bytes in flight per
 * SM: faster on large grids, slower on small ones); 4: the tile build (no
 * rings: 256-thread blocks stage 32 x 16 cells and their halo in shared
 * memory with plain loads while the point-wise operands of each thread's
 * first row are already in flight); 0 (default): the 3-block build. Results
 * agree to FP32 rounding. */
int mfdm_set_blocks_per_sm(mfdm_model* m, int blocks);

/* Times every candidate segment height with both ring builds (2 and 3 blocks
 * per SM), and the tile build, on this handle's model and shots
 * (a few steps each, CUDA events on the handle's stream), keeps the fastest and
 * writes it to *seg_rows (may be NULL). The choice is cached per device, grid
 * shape, PML width, boundary type and shot count, so a second handle of the
 * same shape is not timed again. The timing steps change the state: on return
 * every shot is back at rest at step 0 with its records cleared, as after
 * mfdm_set_shot(m, shot, 1) or mfdm_batch_reset. */
int mfdm_autotune(mfdm_model* m, int* seg_rows);

/* ---- groups of models ---------------------------------------------------
 * Models of different grid sizes (plain or batched handles, one device)
 * stepped together: every step of every model is one node of one captured
 * CUDA graph, the models on parallel branches, so small models fill the GPU
 * together and the host issues one graph launch per 32 steps of all of them.
 * The reference runs one model per process. */
typedef struct mfdm_group mfdm_group;
/* Groups `n` open handles (not owned; they must outlive the group). */
int mfdm_group_open(mfdm_model* const* models, int n, mfdm_group** out);
/* Advances every model by `nsteps` (all must be at the same time index), then
 * synchronises and checks each model's non-finite flag. */
int mfdm_group_step(mfdm_group* g, int nsteps);
/* As mfdm_group_step, reporting the device time of the whole run (ms). */
int mfdm_group_time_steps(mfdm_group* g, int nsteps, float* total_ms);
int mfdm_group_close(mfdm_group* g);

/* ---- adjoint-state gradients ---------------------------------------------
 * The reference has no adjoint. These return the exact gradient of
 * J = sum over receiver samples of residual . record, for a plain handle's
 * current shot started from rest, with respect to the seven coefficient
 * arrays of the model: the discrete adjoint of this library's own RK4 step
 * (transposed stage operators, interface filter and RK4 bookkeeping), with
 * checkpoint-and-recompute time stepping. For an L2 misfit the residual is
 * record - observed. Gradients with respect to vp, vs and rho follow by the
 * chain rule (C11 = C33 = rho vp^2, C13 = rho (vp^2 - 2 vs^2), C55 = rho vs^2). */
typedef struct mfdm_coef_grad {
  double* K;          /* d J / d K                     [nz_f][nx] (any pointer may be NULL) */
  double* rcp_rho_f;  /* d J / d (1 / rho), fluid      [nz_f][nx] */
  double* C11;        /* d J / d C11                   [nz_s][nx] */
  double* C13;
  double* C33;
  double* C55;
  double* rcp_rho_s;  /* d J / d (1 / rho), solid      [nz_s][nx] */
} mfdm_coef_grad;

/* Device memory (bytes) the adjoint may use to keep the stage inputs of whole
 * checkpoint segments during mfdm_adjoint_forward (4 * ckpt_every states per
 * segment; the last segments first), so that the backward pass does not
 * recompute them. 0 (the default): every segment is recomputed from its
 * checkpoint. On a 180 GB B200 an 800x400 model keeps all 4000 steps of a run
 * in about 85 GB. Takes effect with the next mfdm_adjoint_forward. */
int mfdm_adjoint_set_memory(mfdm_model* m, long long bytes);

/* A second checkpoint level for runs whose segments do not fit: with
 * inner_every > 0 (and below ckpt_every) the backward pass re-runs each
 * recomputed segment once keeping a state every inner_every steps, then
 * recomputes and reverses one inner stretch at a time, so it holds
 * ceil(ckpt_every / inner_every) + 4 * inner_every states instead of
 * 4 * ckpt_every, for one more forward pass. 0 (the default): one level.
 * For example 8000 steps of an 8192x4096 model (0.55 GB per state) held
 * 66.6 GB of device memory in all with ckpt_every 200 and inner_every 5. */
int mfdm_adjoint_set_inner(mfdm_model* m, int inner_every);

/* Runs `nsteps` steps of the current shot from rest, storing the state every
 * `ckpt_every` steps (ceil(nsteps / ckpt_every) state copies on the device).
 * The records are read with mfdm_get_records as after mfdm_step. The first
 * call on a handle also assembles the transposed stage operators (lattice
 * probes of the stage kernel; about 2 x 49 stage launches per state array). */
int mfdm_adjoint_forward(mfdm_model* m, int nsteps, int ckpt_every);

/* Back-propagates receiver residuals through the run of the preceding
 * mfdm_adjoint_forward (no other step in between): res_* are
 * [ceil(nsteps / gap)][nx] (NULL = 0), in the mfdm_get_records layout.
 * Recomputes each checkpoint segment once, keeping its stage inputs
 * (4 * ckpt_every state copies; a second such buffer, allocated on first use
 * where memory allows, lets the next segment be recomputed while the current
 * one is reversed). On return the handle is back at rest at step 0. */
int mfdm_adjoint_backward(mfdm_model* m, const float* res_svx, const float* res_svz,
                          const float* res_fp, mfdm_coef_grad* grad);

/* Adds the gradient of the preceding mfdm_adjoint_backward, each value rounded
 * to FP32, to the caller's device buffer `dst` of (2 nz_f + 5 nz_s) x nx floats
 * (K, 1/rho_f, C11, C13, C33, C55, 1/rho_s, each [rows][nx], packed), on
 * `stream` (a cudaStream_t; NULL = legacy default stream) and returns without
 * waiting. The gradient stays on the device: a rank sums its shots into one
 * buffer and the ranks all-reduce it there. No counterpart in the reference,
 * which has no adjoint. */
int mfdm_adjoint_accumulate_grad_f32(mfdm_model* m, float* dst, void* stream);

/* ---- solid only --------------------------------------------------------------
 * calc_type 0 with boundary_type 2: the reference's PmlFs::SolidOnly
 * (include/pml_fs_kernels.cuh:8-307, src/pml_fs_kernels.cu:5-381): an elastic
 * solid filling the grid, a traction-free surface on row 3 (ALM coefficients,
 * src/elements.cu:907-977), CFS-PML left, right and bottom, an explosive source
 * on sx and sz. The receiver row is solid vz on row 3 (src/main.cu:284-300).
 * calc_type 0 with boundary_type 1: Cpml::SolidOnly (include/cpml_kernels.cuh:
 * 8-233, src/cpml_kernels.cu:5-361): CFS-PML on all four sides, no free
 * surface, receiver row 30 (src/main.cu:303-311).
 * The drop-in command line takes this path when the JSON has calc_type 0. */
typedef struct mfdm_solid mfdm_solid;

/* A solid-only model from caller memory: every array [nz][nx] row-major. */
typedef struct mfdm_solid_desc {
  int nx, nz;
  float fpeak, dt;
  int nt, snapshot;
  int npd, npow;
  float thickness, vp_max, rc, beta0;
  int nsrc;
  const int* src_x;
  const int* src_z;
  const float *C11, *C13, *C33, *C55, *rho;
  const float *J, *xi_x, *xi_z, *ze_x, *ze_z;
  int boundary_type;  /* 2 (or 0): free surface on top; 1: CFS-PML on all four
                         sides, Cpml::SolidOnly (include/cpml_kernels.cuh:8-233),
                         the record row is then row 30 (src/main.cu:303-311) */
} mfdm_solid_desc;

int mfdm_solid_open_json(const char* json_path, int device, mfdm_solid** out);
int mfdm_solid_open_desc(const mfdm_solid_desc* d, int device, mfdm_solid** out);
/* Selects source `isrc`, rewinds to step 0 and clears the records; the
 * wavefield is kept unless reset_state (as mfdm_set_shot). */
int mfdm_solid_set_shot(mfdm_solid* m, int isrc, int reset_state);
/* Advances nsteps steps (graph-captured time loop, as mfdm_step). */
int mfdm_solid_step(mfdm_solid* m, int nsteps);
/* As mfdm_solid_step, reporting the device time (ms) of the whole run. */
int mfdm_solid_time_steps(mfdm_solid* m, int nsteps, float* total_ms);
/* Receiver samples [first, first + count) of solid vz on row 3: [count][nx]. */
int mfdm_solid_get_records(mfdm_solid* m, int first, int count, float* solid_vz);
/* One field (MFDM_SOLID_VX .. MFDM_SOLID_SXZ) to a host [nz][nx] array. */
int mfdm_solid_get_field(mfdm_solid* m, int field, float* host);
int mfdm_solid_get_info(const mfdm_solid* m, int* nx, int* nz, int* gap, int* step);
int mfdm_solid_close(mfdm_solid* m);

/* The drop-in command line: `main_debug <model.json> <out_root>`
 * (src/main.cu:58-216). Clears out_root, runs every shot and writes
 * <out_root>/<shot>/record/{solid_vx,solid_vz,fluid_p}.bin and
 * <out_root>/<shot>/snapshot/{solid,fluid}/{vx,vz}/<f>_%06d.bin byte for byte
 * in the reference layout. Returns MFDM_OK or an error code (the CLI exits 1). */
int mfdm_run_cli(const char* json_path, const char* out_root, int device);

/* Snapshots of the command line are drained asynchronously: at a snapshot
 * step the fields are copied on the device into a staging slot and the
 * stepping goes on while a copy stream and a writer thread produce the files.
 * With the environment variable MFDM_SNAPSHOT_PRESSURE=1 the fluid pressure is
 * also written, <shot>/snapshot/fluid/p/p_%06d.bin (listed in the reference's
 * docs/io.md:18, not written by its main.cu). */

/* Every source of the JSON as one batch (mfdm_open_batch with the JSON's
 * fpeak and beta0 for every shot): each shot starts from rest - unlike
 * mfdm_run_cli and the reference, which carry the wavefield from one shot to
 * the next (src/main.cu:94-136) - and all shots step in one launch per RK
 * stage. Writes the same <out_root>/<shot>/ tree per shot. The CLI binary
 * takes this path when MFDM_BATCH=1. */
int mfdm_run_cli_batch(const char* json_path, const char* out_root, int device);

/* ---- stepping without allocating ------------------------------------------
 * No counterpart in the reference. For callers that cannot allocate device
 * memory (a fixed device-memory budget set at start-up, a framework pool that
 * owns the GPU, code where cudaMalloc must not run) but already hold the model
 * and the wavefield on the current device. All arrays below are device
 * pointers, row-major [rows][nx] float32 with row pitch nx; the model arrays
 * are read, the eight state arrays are read and overwritten.
 */
typedef struct mfdm_device_model {
  int nx, nz_f, nz_s;
  float fpeak, dt;
  int npd, npow;
  float thickness, vp_max, rc, beta0;
  int src_x, src_z;               /* source column / fluid row (src_x < 0: none) */
  const float* K;                 /* [nz_f][nx] */
  const float* rho_f;
  const float* C11;               /* [nz_s][nx] */
  const float* C13;
  const float* C33;
  const float* C55;
  const float* rho_s;
  const float* J;                 /* [nz_f+nz_s-1][nx] */
  const float* xi_x;
  const float* xi_z;
  const float* ze_x;
  const float* ze_z;
  float* vx_f;                    /* [nz_f][nx] state, in and out */
  float* vz_f;
  float* p_f;
  float* vx_s;                    /* [nz_s][nx] state, in and out */
  float* vz_s;
  float* sx_s;
  float* sz_s;
  float* sxz_s;
} mfdm_device_model;

/* ---- phase-shift dispersion imaging ----------------------------------------
 * Replaces the reference's post-processing `dispersion_imaging`
 * (tools/test.py:50-98) with a GPU pass over a receiver gather: the real FFT
 * of every trace over time, the phase spectrum conj(S)/|S|, and for every
 * frequency bin w_k = 2 pi k fs / nt (k = 0 .. nt/2) and test velocity
 * c_j = c_min + j dc the normalised stack
 * A[k][j] = |sum_r P[k][r] exp(-i w_k x_r / c_j)| / ntr, all in FP64.
 * Number of test velocities of (c_min, c_max, dc) (numpy.arange(c_min,
 * c_max + dc/2, dc)); 0 for an invalid range. */
int mfdm_dispersion_velocities(double c_min, double c_max, double dc);

/* gather: host [nt][ntr] float32 (the mfdm_get_records layout, traces already
 * selected); offsets: host [ntr] signed source-receiver offsets (m); fs:
 * sampling rate (Hz); amplitude: host [nt/2+1][nv] with nv from
 * mfdm_dispersion_velocities. Allocates its device buffers on `device` and
 * frees them before it returns. */
int mfdm_dispersion_image(const float* gather, int nt, int ntr, const double* offsets, double fs,
                          double c_min, double c_max, double dc, float* amplitude, int device);

/* Size of the library's static device array used by mfdm_step_noalloc; every
 * GPU that loads the library holds it until the process exits. */
#define MFDM_NOALLOC_MAX_BYTES (32u << 20)

/* Steps time indices it .. it + nsteps - 1 of `dm` on `stream` (a cudaStream_t,
 * NULL = legacy default stream) and returns after the stream has finished.
 * Allocates nothing: the coefficient blocks, RK stage buffers, accumulator,
 * ADE memory and tables live in one static device array of
 * MFDM_NOALLOC_MAX_BYTES; models that need more are rejected with
 * MFDM_ERR_ARG (the size depends on the grid only: calls of many steps run
 * them in chunks of 1024 with a fixed Ricker table). A source cell outside the
 * fluid grid is rejected (src_x < 0: no source). The Ricker and PML tables come
 * from the same host functions as an open handle's, so the results are
 * bit-identical to mfdm_step on the same model. The first call on a device
 * resolves that array's address and configures the kernels there, so make it
 * before any stream capture; after cudaDeviceReset of that device, do not call
 * it again in the same process. Calls share the array and it keeps the last
 * call's contents: the ADE memory carries from one call to the next, so start
 * a run with it == 0 (which clears it) and continue one model with consecutive
 * time indices; calls that overlap on the GPU race. A pipeline wait that times
 * out returns MFDM_ERR_CUDA and leaves the state arrays undefined. No receiver
 * buffer: read the state arrays. */
int mfdm_step_noalloc(const mfdm_device_model* dm, int it, int nsteps, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MFDM_H */
