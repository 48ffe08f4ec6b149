/*
 * fdtd_b200.h -- C ABI of the B200 (sm_100a) FDTD time-step engine.
 *
 * Drop-in for the reference's CUDA backend boundary
 * (js_fdtd/src/backends/cuda/native/fdtd_cuda.h:12-63, driven by
 * js_fdtd/src/backends/cuda/native/binding.cpp:174-185 and
 * js_fdtd/src/backends/cuda/cudaBackend.js:183-289).  Every legacy entry point
 * of that header is exported under the same name and signature; the rest is a
 * superset: a handle per simulation, FP64 uploads, several sources and probes,
 * the far-field DFT on the device, material-table (FP32) problems, many
 * problems advanced in one launch, and watchdog status codes.
 *
 * Plain pointers and sizes only.  Host buffers are borrowed for the duration
 * of a call and copied to the device inside it (binding.cpp:51-60 semantics).
 * Every call is synchronous with respect to the host; a handle owns one CUDA
 * stream and must not be used from two host threads at once.
 *
 * Index conventions are those of the reference's problem object
 * (js_fdtd/src/backends/CONTRACT.md:15-57): flat, row-major, 0-based,
 * k fastest; component extents Hx (nx+1,ny,nz) Hy (nx,ny+1,nz) Hz (nx,ny,nz+1)
 * Ex (nx,ny+1,nz+1) Ey (nx+1,ny,nz+1) Ez (nx+1,ny+1,nz).
 */
#ifndef FDTD_B200_H
#define FDTD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  FDTD_OK / FDTD_ERR keep the reference's values (fdtd_cuda.h:12-13). */
#define FDTD_OK 0
#define FDTD_ERR 1
#define FDTD_ERR_BADARG 2     /* argument failed validation; nothing was changed */
#define FDTD_ERR_OOM 3        /* device allocation failed */
#define FDTD_ERR_CUDA 4       /* a CUDA runtime call failed */
#define FDTD_ERR_NONFINITE 5  /* the watchdog saw a NaN/Inf port sample; see fdtd_status */
#define FDTD_ERR_STATE 6      /* call not valid in the handle's current state */

/* Arithmetic of a problem's fields. */
#define FDTD_PREC_F64 0       /* FP64 fields, 18 per-cell coefficient arrays (the reference's layout) */
#define FDTD_PREC_F32 1       /* FP32 fields, 18 per-cell coefficient arrays */
#define FDTD_PREC_F32_TABLE 2 /* FP32 fields, per-component material ids into coefficient tables */

/* Field ids (fdtd_cuda.cu read_field order). */
#define FDTD_HX 0
#define FDTD_HY 1
#define FDTD_HZ 2
#define FDTD_EX 3
#define FDTD_EY 4
#define FDTD_EZ 5

/* Legacy problem size (fdtd_cuda.h:15-19).  Spacings are float there. */
typedef struct {
  int nx, ny, nz;
  float dx, dy, dz, dt;
  int numberOfTimeSteps;
} FdtdDims;

/* Problem size with FP64 spacings and the field arithmetic. */
typedef struct {
  int nx, ny, nz;
  double dx, dy, dz, dt;
  int numberOfTimeSteps;
  int precision; /* FDTD_PREC_* */
  int device;    /* CUDA device ordinal */
} FdtdConfig;

typedef struct fdtd_ctx fdtd_ctx;

/* ---- legacy global-context API (fdtd_cuda.h:21-63), same names and meaning ---- */

/* Last error message of any failing call on this thread (never NULL). fdtd_cuda.h:22 */
const char* fdtd_last_error(void);
/* Number of CUDA devices; 0 and FDTD_OK when there is no driver. fdtd_cuda.h:25 */
int fdtd_device_count(int* count);
/* Frees any previous global problem and allocates a new FP32 one. fdtd_cuda.h:28 */
int fdtd_init(const FdtdDims* d);
/* Uploads coefficient `which` (0..17 in the order of cudaBackend.js:53-60:
 * Cexe Cexhz Cexhy Ceye Ceyhx Ceyhz Ceze Cezhy Cezhx Chxh Chxey Chxez Chyh Chyez Chyex
 * Chzh Chzex Chzey). fdtd_cuda.h:31 */
int fdtd_upload_coeff(int which, const float* host, int n);
/* One CPML face, faceId 0..5 = xn xp yn yp zn zp; slots as cudaBackend.js:76-116
 * (x: hyx hzx eyx ezx, y: hxy hzy ezy exy, z: hxz hyz exz eyz). fdtd_cuda.h:36 */
int fdtd_upload_cpml(int faceId, int nc, const float* b_e, const float* a_e, const float* b_m,
                     const float* a_m, const float* CPsi0, int n0, const float* CPsi1, int n1,
                     const float* CPsi2, int n2, const float* CPsi3, int n3, int m_start, int e_start,
                     int ascending);
/* Adds a lumped voltage source (dir 0=x 1=y 2=z). fdtd_cuda.h:43 */
int fdtd_upload_vsource(int dir, const int* idx, const float* coef, int count, const float* waveform,
                        int nSteps);
/* Adds a sampled-voltage probe V = Csvf * sum E[idx]. fdtd_cuda.h:47 */
int fdtd_upload_svoltage(int dir, const int* idx, int count, float Csvf);
/* Adds a sampled-current probe as three weighted gather lists. fdtd_cuda.h:50 */
int fdtd_upload_scurrent(const int* hxIdx, const float* hxW, int hxN, const int* hyIdx, const float* hyW,
                         int hyN, const int* hzIdx, const float* hzW, int hzN);
/* Runs steps [tsStart, tsStart+count); svOut/siOut (may be NULL) receive the
 * first voltage / current probe per step. fdtd_cuda.h:57 */
int fdtd_run_batch(int tsStart, int count, float* svOut, float* siOut);
/* Copies field `which` (0=Hx..5=Ez) to the host. fdtd_cuda.h:60 */
int fdtd_read_field(int which, float* host, int n);
/* Frees the global problem. fdtd_cuda.h:63 */
void fdtd_destroy(void);

/* ---- handle API (superset) ---- */

/* Allocates a problem on cfg->device.  Fields, Psi and accumulators start at zero. */
int fdtd_create(const FdtdConfig* cfg, fdtd_ctx** out);
/* Frees everything the handle owns; NULL is ignored. */
void fdtd_free(fdtd_ctx* ctx);

/* FP64 / FP32 per-cell coefficient array `which` (same ids as fdtd_upload_coeff).
 * The host array is FP64 and is rounded once when the problem is FP32. */
int fdtd_ctx_upload_coeff(fdtd_ctx* ctx, int which, const double* host, long n);

/* One CPML face (js_fdtd/src/cpml.js:147-448): 1-D b/a profiles of length nc,
 * CPsi slot arrays in the reference's Psi layouts, and the first H / E index of
 * the face along its axis.  kappa_e / kappa_m (length nc, may be NULL for the
 * per-cell problems) are needed by FDTD_PREC_F32_TABLE problems, whose
 * coefficient tables carry no kappa division.  An FP64 problem whose
 * coefficients came from fdtd_ctx_build_material passes no CPsi (all four
 * pointers NULL, counts 0) and the kappa profiles instead: the device then
 * takes CPsi from the coefficients and divides the face's band of them by
 * kappa, as cpml.js:212-243 does, once per face, in the order the faces are
 * uploaded. */
int fdtd_ctx_upload_cpml(fdtd_ctx* ctx, int faceId, int nc, const double* b_e, const double* a_e,
                         const double* b_m, const double* a_m, const double* kappa_e, const double* kappa_m,
                         const double* CPsi0, long n0, const double* CPsi1, long n1, const double* CPsi2,
                         long n2, const double* CPsi3, long n3, int m_start, int e_start);

/* Lumped voltage source (sources.js:271-288): E_dir[idx[n]] += coef[n] * wave[ts]
 * after the electric CPML.  idx must list an axis-aligned box of cells of
 * component dir in the reference's createLinearIndexList order (k outer, j,
 * i inner); wave has one value per step (voltage_per_e_field). */
int fdtd_ctx_add_vsource(fdtd_ctx* ctx, int dir, const int* idx, const double* coef, int count,
                         const double* wave, int nSteps);

/* Sampled voltage (sampling.js:295-307): V[ts] = Csvf * (sum over idx in order). */
int fdtd_ctx_add_svoltage(fdtd_ctx* ctx, int dir, const int* idx, int count, double Csvf);

/* Sampled current (sampling.js:204-245) as ONE ordered gather list:
 * I[ts] = sum_n w[n] * H_comp[n][idx[n]], summed in list order from zero, with
 * comp 0=Hx 1=Hy 2=Hz and the reference's signs folded into w. */
int fdtd_ctx_add_scurrent(fdtd_ctx* ctx, const int* comp, const int* idx, const double* w, int count);

/* Running NF-FF DFT on the Huygens box (farfield.js:28-78,90-248).  li..uk are
 * the reference's 1-based box bounds.  Phasors cos/-sin of w*dt*(ts+0.5) and
 * w*dt*(ts+1) are evaluated here in FP64, w = 2*pi*f. */
int fdtd_ctx_setup_farfield(fdtd_ctx* ctx, int nFreq, const double* freqs, int li, int lj, int lk, int ui,
                            int uj, int uk);

/* Material-table problem (FDTD_PREC_F32_TABLE): one uint8 id per cell and
 * component selects a row of that component's coefficient table
 * (rows x 3: self, first curl, second curl coefficient, all without kappa).
 * comp order Ex Ey Ez Hx Hy Hz; curl order as the per-cell arrays
 * (Ex: Cexe Cexhz Cexhy, ..., Hz: Chzh Chzex Chzey). */
int fdtd_ctx_upload_material(fdtd_ctx* ctx, int comp, const unsigned char* ids, long n, const double* table,
                             int rows);

/* Coefficients built on the device from the material grid, for
 * FDTD_PREC_F32_TABLE problems (ids and tables) and FDTD_PREC_F64 problems (the
 * 18 per-cell arrays, bit-identical to the reference's arithmetic, before the
 * CPML kappa division, which fdtd_ctx_upload_cpml then applies)
 * (materials.js:21-332 + coefficients.js:22-116): `mat` holds one type id per
 * cell (nx*ny*nz, k fastest; 1-based ids as materials.js stores them), `props`
 * has 4 values per type id 0..ntypes-1 (eps_r, mu_r, sigma_e, sigma_m, with
 * materials.js:96-101's zero replacements already applied), `plates` has 7 ints
 * per zero-thickness PEC plate box (component 0=Ex 1=Ey 2=Ez, then inclusive
 * i0 i1 j0 j1 k0 k1 of that component array) applied in order with conductivity
 * plate_sigma[q] (materials.js:253-332).  At most 48 type ids and 64 plates. */
int fdtd_ctx_build_material(fdtd_ctx* ctx, const unsigned char* mat, long ncells, int ntypes, const double* props,
                            int nplates, const int* plates, const double* plate_sigma);

/* Gives `count` cells of component comp (API order Ex Ey Ez Hx Hy Hz) their own
 * coefficient triples (self, curl1, curl2), e.g. the lumped-source cells of
 * coefficients.js:158-207: new table rows for FDTD_PREC_F32_TABLE problems,
 * the three per-cell arrays of comp for FDTD_PREC_F64 problems. */
int fdtd_ctx_override_material(fdtd_ctx* ctx, int comp, const int* idx, const double* triples, int count);

/* Reads back a component's ids and its coefficient table (FP64, rows x 3). */
int fdtd_ctx_read_material(fdtd_ctx* ctx, int comp, unsigned char* ids, long n, double* table, int* rows);

/* Runs `count` steps from the handle's current step.  Checks the watchdog at
 * the end and returns FDTD_ERR_NONFINITE if a port sample went non-finite. */
int fdtd_ctx_run(fdtd_ctx* ctx, int count);
/* Launch shape of the two step kernels: each thread walks `x_planes_per_thread`
 * consecutive x planes of one (j, k) column; a block is `width` columns along k
 * (fdtd_ctx_set_block_width: 32, the default, or 16, when a warp spans two
 * rows, which wastes fewer lanes when nz + 1 is not a multiple of 32) by
 * `block_rows` (1, 2, 4, 8 or 16) along j, in whole warps of at most 256
 * threads (checked at the next run).  Any shape gives the same results; the
 * autotuner (special-topics_b200/autotune.py) picks the fastest per grid. */
int fdtd_ctx_set_tiling(fdtd_ctx* ctx, int x_planes_per_thread, int block_rows);
int fdtd_ctx_get_tiling(const fdtd_ctx* ctx, int* x_planes_per_thread, int* block_rows);
int fdtd_ctx_set_block_width(fdtd_ctx* ctx, int threads_along_k);
int fdtd_ctx_get_block_width(const fdtd_ctx* ctx, int* threads_along_k);
/* How the interior loop of the step kernels fetches its planes: 1 or 2 =
 * that many planes ahead into registers; 3 or 4 (material-table problems) =
 * that many planes staged through shared memory, word by word; 5
 * (material-table problems, 32-wide blocks) = the H half-step's rows staged
 * through a shared-memory ring by bulk copies on mbarriers.  Same results
 * in every mode; the autotuner picks among 1-4. */
int fdtd_ctx_set_prefetch(fdtd_ctx* ctx, int planes);
/* fdtd_ctx_run that also reports the device time (ms) between CUDA events
 * recorded on the handle's stream before the first and after the last launch. */
int fdtd_ctx_run_timed(fdtd_ctx* ctx, int count, float* ms);
/* Runs `count` steps one at a time with CUDA events around every launch and
 * returns the mean duration (ms) of the H, mid-step, E and epilogue kernels. */
int fdtd_ctx_profile_kernels(fdtd_ctx* ctx, int count, double* avg_ms);
/* Current step index (number of completed steps). */
int fdtd_ctx_step(const fdtd_ctx* ctx);
/* Watchdog: *code = FDTD_OK or FDTD_ERR_NONFINITE, *step = first bad step or -1. */
int fdtd_status(fdtd_ctx* ctx, int* code, int* step);

/* ---- batches: many handles advanced together (no counterpart in the reference,
 * which runs one problem per process through its global context,
 * fdtd_cuda.cu:44-118; used for sweeps over antenna variants) ---- */
typedef struct fdtd_batch fdtd_batch;

/* Groups `count` handles of one device and one precision.  The batch owns no
 * member: members stay valid handles (readbacks, fdtd_status, their own runs)
 * and must outlive the batch.  By default each step of fdtd_batch_run is four
 * launches for the whole batch: H over a tile list spanning every member, the
 * mid-step kernel, E over the tile list, and the far-field/port epilogue
 * (fdtd_batch_set_streams selects the member-kernel mode instead). */
int fdtd_batch_create(fdtd_ctx* const* members, int count, fdtd_batch** out);
void fdtd_batch_free(fdtd_batch* batch);
int fdtd_batch_size(const fdtd_batch* batch);
/* Launch shape shared by all members: x planes per thread and block rows as in
 * fdtd_ctx_set_tiling, prefetch depth as in fdtd_ctx_set_prefetch, and `group`:
 * 0 = one block per tile; g > 0 = a persistent grid (as many blocks as are
 * resident on the device) whose blocks claim g consecutive tiles at a time from
 * a device counter.  Results do not depend on the shape.  x_planes_per_thread
 * may be 1..1024 whatever the members' depth: a member with nx + 1 planes or
 * fewer than it gets one chunk per column, and fdtd_batch_get_tiling reports
 * the value as set, not the per-member value in effect. */
int fdtd_batch_set_tiling(fdtd_batch* batch, int x_planes_per_thread, int block_rows, int prefetch, int group);
int fdtd_batch_get_tiling(const fdtd_batch* batch, int* x_planes_per_thread, int* block_rows, int* prefetch,
                          int* group);
/* Member-kernel mode: streams = S > 0 runs each member's own step kernels
 * (those of fdtd_ctx_run, with the batch's launch shape), the members spread
 * over S worker streams inside one CUDA graph, all steps of a graph for one
 * member before the next member of its stream (so a member's arrays stay in L2
 * from one step to the next).  streams = 0 (default) is the tile-list mode.
 * Results are identical in both modes.  S <= 32. */
int fdtd_batch_set_streams(fdtd_batch* batch, int streams);
/* Block width along k of the batch's step launches (16 or 32), as
 * fdtd_ctx_set_block_width. */
int fdtd_batch_set_block_width(fdtd_batch* batch, int threads_along_k);
int fdtd_batch_get_block_width(const fdtd_batch* batch, int* threads_along_k);
int fdtd_batch_get_streams(const fdtd_batch* batch, int* streams);
/* Grouped mode (used when streams is 0): members > 0 carries that many
 * members' parameter blocks (at most 22) as the parameter of one launch, in
 * member order, so the step kernels read them from the constant bank as a
 * single problem's launch does; the group launches of a half-step run side by
 * side on worker streams.  0 (default) = the tile-list or persistent launches
 * of fdtd_batch_set_tiling.  Results do not depend on the mode. */
int fdtd_batch_set_members_per_launch(fdtd_batch* batch, int members);
int fdtd_batch_get_members_per_launch(const fdtd_batch* batch, int* members);
/* Runs `count` steps of every member.  All members must be at the same step and
 * have `count` steps left.  Returns FDTD_ERR_NONFINITE naming the first member
 * whose watchdog fired. */
int fdtd_batch_run(fdtd_batch* batch, int count);
int fdtd_batch_run_timed(fdtd_batch* batch, int count, float* ms);
/* Per-kernel mean durations (ms) of the batch's H, mid-step, E and epilogue
 * launches per step (member-kernel mode: each member timed alone, summed over
 * the members). */
int fdtd_batch_profile_kernels(fdtd_batch* batch, int count, double* avg_ms);

/* Whole probe traces, FP64, one value per step (first `n` steps). kind 0 = voltage, 1 = current. */
int fdtd_ctx_read_trace(fdtd_ctx* ctx, int kind, int probe, double* out, int n);
/* Field `which` as FP64 (FP32 problems are widened). */
int fdtd_ctx_read_field(fdtd_ctx* ctx, int which, double* host, long n);
/* CPML Psi slot of a face, as FP64. */
int fdtd_ctx_read_psi(fdtd_ctx* ctx, int faceId, int slot, double* host, long n);
/* Far-field accumulator `array` (0..23 in the order cjyxp cjzxp cjyxn cjzxn cjxyp cjzyp
 * cjxyn cjzyn cjxzp cjyzp cjxzn cjyzn cmyxp cmzxp cmyxn cmzxn cmxyp cmzyp cmxyn cmzyn
 * cmxzp cmyzp cmxzn cmyzn), laid out [freq][point] like farfield.js:55. */
int fdtd_ctx_read_farfield(fdtd_ctx* ctx, int array, double* re, double* im, long n);

/* Time-blocked surface DFT of an FP32 problem: the epilogue buffers each
 * step's surface samples and every `steps` steps (and at the end of each run)
 * they are accumulated at once, so the accumulators are read and written once
 * per block instead of once per step.  0 (default) = every step; FP64
 * problems keep the per-step form (their summation order is the reference's).
 * Results match the per-step form to FP32 rounding. */
int fdtd_ctx_set_dft_block(fdtd_ctx* ctx, int steps);

/* Checkpoint / restore (the reference has none): the evolving state of a
 * handle -- fields, Psi, port traces, far-field accumulators, watchdog and
 * step -- to and from a caller buffer of fdtd_ctx_state_size bytes.  The
 * state carries a 64-bit digest of everything the handle was set up with:
 * grid, cell sizes, dt, step count, precision and the data of every set-up
 * call (coefficients or material grid and tables, CPML profiles and CPsi,
 * sources, probes, far-field frequencies and box), in call order.  A state
 * loads only into a handle whose digest matches, that is one set up by the
 * same calls with the same data; any other fails with FDTD_ERR_BADARG.
 * Stepping on from a loaded state gives the results of stepping on from the
 * saved one. */
int fdtd_ctx_state_size(fdtd_ctx* ctx, long long* bytes);
int fdtd_ctx_save_state(fdtd_ctx* ctx, void* buf, long long bytes);
int fdtd_ctx_load_state(fdtd_ctx* ctx, const void* buf, long long bytes);

/* Far-field accumulator arithmetic of an FP32 problem: 0 = FP64 (default),
 * 1 = Kahan-compensated FP32 pairs (same 8 bytes per value).  Readback
 * returns FP64 either way.  Set before the first step; FP64 problems keep
 * FP64.  No counterpart in the reference (its accumulators are Float64Array). */
int fdtd_ctx_set_dft_accumulator(fdtd_ctx* ctx, int kahan_fp32);

/* The E update at the x = max wall.  The reference's updateE runs Ey and Ez
 * up to i = nx inclusive (js_fdtd/assembly/fdtd_kernels.ts:159,185 with the
 * worker range end nxp1, js_fdtd/src/fdtdWorker.js:22-30) and there reads one
 * plane past the Hz and Hy arrays, which in its shared memory are Ex(i=0) and
 * the start of Hz: a coupling of the two x walls that grows without bound at
 * late times (js_fdtd/scenarios/ifa-matlab-7000.json:3).  The MATLAB original
 * updates Ey, Ez only for i < nx (fdtd_solve_Ch9_ex9a_12032026.m.txt:2095-2106),
 * a PEC wall.
 *   wall = 0: the reference's reads (default for FDTD_PREC_F64: bit parity);
 *   wall = 1: Ey and Ez at i = nx are never updated and stay zero (default for
 *             the FP32 precisions, whose rounding would otherwise seed the
 *             growing mode some nine orders of magnitude above FP64's).
 * May be changed between runs. */
int fdtd_ctx_set_x_wall(fdtd_ctx* ctx, int wall);
int fdtd_ctx_get_x_wall(const fdtd_ctx* ctx, int* wall);

/* Far-field post-processing on the device from the handle's accumulators
 * (farfield.js:257-607): radp[f] = radiated power at frequency f, and the
 * directivity components d_theta / d_phi [nFreq][nang] towards the nang
 * directions (theta[a], phi[a]) in radians (nang may be 0). */
int fdtd_ctx_farfield_post(fdtd_ctx* ctx, const double* theta, const double* phi, int nang, double* radp,
                           double* d_theta, double* d_phi);

/* Direct time-to-frequency transform on the device (dft.js:17-38):
 * X(f) = dt * sum_n x[n] exp(-j 2 pi f ((n+1) dt + shift)), FP64. */
int fdtd_dft(const double* x, int N, double dt, const double* freqs, int M, double shift, double* re,
             double* im);

/* The same transform as fdtd_dft, for callers that must not allocate device
 * memory: a host whose device memory is owned by another component's pool or
 * budget, or a loop that cannot afford cudaMalloc/cudaFree, which may
 * synchronise the whole device.  No counterpart in the reference.
 * Nothing is allocated or freed: inputs and outputs are staged through one
 * fixed device array of 45,056 doubles (352 KiB), which every GPU that loads
 * the library holds until the process exits.  Limits: N <= 32768 samples and
 * M <= 4096 frequencies; larger calls fail with FDTD_ERR_BADARG.  The first
 * call on a device looks up that array's address, so make that first call
 * before any stream capture.  The address is kept for the life of the process:
 * it assumes the device's primary context does too (a host that resets the
 * device with cudaDeviceReset must not call this entry point afterwards).
 * All calls share the array: calls that overlap on
 * the GPU (from several host threads) race and must be serialised by the
 * caller.  Each call writes every value it reads, so no call sees another's. */
int fdtd_dft_noalloc(const double* x, int N, double dt, const double* freqs, int M, double shift, double* re,
                     double* im);

/* ---- learned early stop: a 1-D convolutional network with an MLP head that
 * reads the first steps of the port transient (no counterpart in the
 * reference, whose runs always take numberOfTimeSteps steps, index.js:54-60).
 * Weights enter the arithmetic as BF16 copies of FP32 master values, biases
 * as FP32; every sum accumulates in FP32.
 *
 * Data layout: a sample is `in_length` x `in_channels` values, time major
 * (channel fastest).  Layers: `conv_layers` convolutions (kernel `kernel`,
 * stride `stride`, zero padding kernel/2, ReLU) from in_channels to `channels`
 * channels, the flattened result (time major, channel fastest), `mlp_layers`
 * dense layers of `mlp_width` with ReLU, and a linear head of `out_dim`.
 * Flat parameter order: per convolution W[cout][kernel][cin] then b[cout];
 * per dense layer (the head last) W[out][in] then b[out]. ---- */
typedef struct fdtd_es_net fdtd_es_net;

typedef struct {
  int in_channels, in_length;
  int conv_layers, channels, kernel, stride;
  int mlp_layers, mlp_width;
  int out_dim;
  int max_batch; /* largest batch any call passes */
  int device;
} FdtdEsConfig;

int fdtd_es_create(const FdtdEsConfig* cfg, fdtd_es_net** out);
void fdtd_es_free(fdtd_es_net* net);
int fdtd_es_param_count(const fdtd_es_net* net, long* count);
/* Seeded initialisation: every weight and bias uniform in +-1/sqrt(fan_in). */
int fdtd_es_init_params(fdtd_es_net* net, unsigned long long seed);
/* FP32 master parameters; setting them also resets the optimiser state. */
int fdtd_es_set_params(fdtd_es_net* net, const float* params, long count);
int fdtd_es_get_params(fdtd_es_net* net, float* params, long count);
/* Forward pass of `batch` samples from host memory; y is batch x out_dim. */
int fdtd_es_forward(fdtd_es_net* net, const float* x, int batch, float* y);
/* Loss L = (1/batch) sum_b sum_o w[o] (y[b][o] - target[b][o])^2 and its
 * gradient with respect to the parameters (grad may be NULL). */
int fdtd_es_loss_grad(fdtd_es_net* net, const float* x, const float* target, const float* w, int batch,
                      float* loss, float* grad, long count);
/* Keeps a training set resident on the device: n samples, targets n x out_dim. */
int fdtd_es_set_data(fdtd_es_net* net, const float* x, const float* target, long n);
/* Adam (decoupled weight decay) over the resident set: `epochs` passes of
 * minibatches of `batch` in a seeded shuffled order (a last partial batch is
 * dropped); epoch_loss[e] = mean minibatch loss of epoch e (may be NULL). */
int fdtd_es_train(fdtd_es_net* net, int epochs, int batch, const float* w, float lr, float beta1, float beta2,
                  float eps, float weight_decay, unsigned long long seed, float* epoch_loss);
/* Network input built on the device from the port traces of handles (for
 * handle b: channel 0 = voltage probe 0, channel 1 = current probe 0, over
 * steps [0, in_length * decim), each value the mean of `decim` consecutive
 * steps, each channel divided by its largest magnitude; scales[2b] and
 * scales[2b+1] receive those divisors, 1 for an all-zero channel).  Needs
 * in_channels == 2 and every handle at step >= in_length * decim.
 * fdtd_es_member_inputs returns the inputs (x: count x in_length x 2, may be
 * NULL); fdtd_es_predict_members runs the forward pass on them (y: count x out_dim). */
int fdtd_es_member_inputs(fdtd_es_net* net, fdtd_ctx* const* members, int count, int decim, float* scales,
                          float* x);
int fdtd_es_predict_members(fdtd_es_net* net, fdtd_ctx* const* members, int count, int decim, float* scales,
                            float* y);

#ifdef __cplusplus
}
#endif
#endif /* FDTD_B200_H */
