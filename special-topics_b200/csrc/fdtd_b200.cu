// fdtd_b200.cu -- host side of the C ABI declared in include/fdtd_b200.h:
// problem handles, uploads with validation, the per-step launch sequence
// (captured into a CUDA graph per batch of steps), readbacks and the legacy
// global-context entry points of js_fdtd/src/backends/cuda/native/fdtd_cuda.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <string>
#include <vector>

#include "../../include/fdtd_b200.h"
#include "fdtd_common.cuh"
#include "fdtd_material.cuh"
#include "fdtd_step.cuh"
#include "fdtd_batch.cuh"
#include "fdtd_ffpost.cuh"
#include "fdtd_internal.h"

#include <map>
#include <mutex>
#include <utility>

using namespace fdtd;

static thread_local char g_err[512] = "no error";

static int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int fdtd_internal_fail(int code, const char* msg) { return fail(code, "%s", msg); }

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return fail(FDTD_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

namespace {

struct HostFace {
  bool present = false;
  int nc = 0, m_start = 0, e_start = 0;
  void* prof[4] = {};   // b_e a_e b_m a_m (field type)
  float* inv_k[2] = {};  // 1/kappa_e, 1/kappa_m (table problems)
  void* psi[4] = {};
  void* cpsi[4] = {};
  long long n[4] = {};
};

struct HostSource {
  SourceBox box;
  int count;
  void* cs;
  void* wave;
};

struct HostVProbe {
  int comp, count;
  int* idx;
  double csvf;
};

struct HostIProbe {
  int count;
  int* comp;
  int* idx;
  double* w;
};

}  // namespace

// CUDA graphs of whole runs, keyed by their step count.  A run of `count`
// steps replays graphs of at most the handle's cap (kMaxGraphNodes over the
// launches one step takes) and one of the remainder; every graph a run needs
// is captured before the run's first launch, so no capture falls inside a
// timed region.  A handful of counts is kept (early-stop runs advance in
// checkpoints of a few different lengths).
struct RunGraphs {
  std::vector<std::pair<int, cudaGraphExec_t>> g;
  void clear() {
    for (auto& e : g) cudaGraphExecDestroy(e.second);
    g.clear();
  }
};

struct fdtd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int prec = FDTD_PREC_F64;
  size_t esz = 8;  // bytes per field value
  int nx = 0, ny = 0, nz = 0, nsteps = 0;
  double dx = 0, dy = 0, dz = 0, dt = 0;
  int ts = 0;  // completed steps
  long long ncomp[6] = {};  // Hx Hy Hz Ex Ey Ez element counts
  void* fields = nullptr;   // contiguous Hx..Ez (+ slack)
  void* coef[18] = {};
  bool coef_set[18] = {};
  bool coef_device = false;     // FP64 coefficients built by fdtd_ctx_build_material
  bool kappa_done[6] = {};      // face whose CPML band of them was divided by kappa on the device
  // material-table problem
  unsigned char* ids[6] = {};
  bool ids_set[6] = {};
  std::vector<float> table[6];
  std::vector<double> rows64[6];  // the same rows in FP64 (rows x 3), for overrides and readback
  float* d_tab = nullptr;      // [6][kTableRows] float4 rows (self, curl1, curl2, 0), field order
  float* d_invk[6] = {};       // 1/kappa per axis position: E x y z, H x y z
  bool table_dirty = true;
  TableCoef tcoef{};
  HostFace face[6];
  std::vector<HostSource> src;
  std::vector<HostVProbe> vprobe;
  std::vector<HostIProbe> iprobe;
  double* V = nullptr;  // traces
  double* I = nullptr;
  int nv_alloc = -1, ni_alloc = -1;
  // far field
  int nFreq = 0;
  int li = 0, lj = 0, lk = 0, ui = 0, uj = 0, uk = 0;
  double* ph = nullptr;
  double* acc = nullptr;
  std::vector<double> ffreq;  // far-field frequencies (Hz)
  int acc_kahan = 0;          // FP32 problems: compensated FP32 accumulator pairs instead of FP64
  int dft_block = 0;          // FP32 problems: steps per time block of the surface DFT (0: every step)
  int x_wall = 0;             // 1: Ey, Ez at i = nx stay zero (see fdtd_ctx_set_x_wall)
  float* dft_samples = nullptr;
  int* d_dft_done = nullptr;
  long long ffsz[3] = {};
  long long ffoff[24] = {};
  void* ex0b = nullptr;
  int* d_ts = nullptr;
  int* d_status = nullptr;
  // launch shape of the step kernels: x planes per thread, thread rows per block
  int ichunk = 1, block_rows = 8, prefetch = 1;
  int block_w = 32;   // threads of a block along k (32: a warp is one row; 16: a warp spans two rows)
  // graph cache
  RunGraphs graphs;
  bool dirty = true;
  std::vector<void*> owned;  // every device allocation
  // Running digest of everything the handle was set up with: shape, spacing,
  // dt, step count, precision and the arguments of every upload call in call
  // order.  A saved state carries it and loads only where it matches.
  unsigned long long setup_digest = 0x6a09e667f3bcc908ULL;
};

namespace {

int dalloc(fdtd_ctx* c, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(FDTD_ERR_OOM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
  }
  c->owned.push_back(*p);
  // Zero on the handle's stream and wait: later uploads may use either stream,
  // and the zeroing must not land after them.
  e = cudaMemsetAsync(*p, 0, bytes, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, "zeroing a new buffer: %s", cudaGetErrorString(e));
  return FDTD_OK;
}

void dfree(fdtd_ctx* c, void* p) {
  if (!p) return;
  auto it = std::find(c->owned.begin(), c->owned.end(), p);
  if (it != c->owned.end()) c->owned.erase(it);
  cudaFree(p);
}

// Copy on the handle's stream and wait.  Every set-up copy goes through here so
// that it is ordered with the zeroing in dalloc and with the kernels, which all
// run on that (non-blocking) stream.
cudaError_t xfer(fdtd_ctx* c, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e;
}

// Host FP64 array -> device array of the problem's field type.
int upload_real(fdtd_ctx* c, void* dst, const double* src, long long n) {
  if (n <= 0) return FDTD_OK;
  if (c->esz == 8) {
    CK(cudaMemcpyAsync(dst, src, n * 8, cudaMemcpyHostToDevice, c->stream));
  } else {
    std::vector<float> tmp(n);
    for (long long q = 0; q < n; q++) tmp[q] = (float)src[q];
    CK(cudaMemcpyAsync(dst, tmp.data(), n * 4, cudaMemcpyHostToDevice, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return FDTD_OK;
}

int read_real(fdtd_ctx* c, const void* srcdev, double* dst, long long n) {
  if (n <= 0) return FDTD_OK;
  if (c->esz == 8) {
    CK(cudaMemcpyAsync(dst, srcdev, n * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  } else {
    std::vector<float> tmp(n);
    CK(cudaMemcpyAsync(tmp.data(), srcdev, n * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (long long q = 0; q < n; q++) dst[q] = tmp[q];
  }
  return FDTD_OK;
}

// Coefficient id -> (component, count) in cudaBackend.js:53-60 order.
long long coef_count(const fdtd_ctx* c, int which) {
  static const int comp_of[18] = {3, 3, 3, 4, 4, 4, 5, 5, 5, 0, 0, 0, 1, 1, 1, 2, 2, 2};
  return c->ncomp[comp_of[which]];
}

void* field_ptr(const fdtd_ctx* c, int which) {
  char* base = (char*)c->fields;
  long long off = 0;
  for (int q = 0; q < which; q++) off += c->ncomp[q];
  return base + off * c->esz;
}

// Expected Psi slot sizes (cpml.js:147-448) for face f with nc cells.
void psi_sizes(const fdtd_ctx* c, int f, int nc, long long out[4]) {
  const long long nx = c->nx, ny = c->ny, nz = c->nz, X = nx + 1, Y = ny + 1, Z = nz + 1;
  if (f / 2 == 0) {
    out[0] = nc * Y * nz; out[1] = nc * ny * Z; out[2] = nc * ny * Z; out[3] = nc * Y * nz;
  } else if (f / 2 == 1) {
    out[0] = X * nc * nz; out[1] = nx * nc * Z; out[2] = X * nc * nz; out[3] = nx * nc * Z;
  } else {
    out[0] = X * ny * nc; out[1] = nx * Y * nc; out[2] = nx * Y * nc; out[3] = X * ny * nc;
  }
}

void invalidate(fdtd_ctx* c) {
  c->dirty = true;
  c->table_dirty = true;
  c->graphs.clear();
}

template <typename T>
Face<T> dev_face(const HostFace& h) {
  Face<T> f{};
  if (!h.present) return f;
  f.nc = h.nc;
  f.m_start = h.m_start;
  f.e_start = h.e_start;
  f.b_e = (const T*)h.prof[0];
  f.a_e = (const T*)h.prof[1];
  f.b_m = (const T*)h.prof[2];
  f.a_m = (const T*)h.prof[3];
  f.inv_ke = h.inv_k[0];
  f.inv_km = h.inv_k[1];
  for (int s = 0; s < 4; s++) {
    f.psi[s] = (T*)h.psi[s];
    f.cpsi[s] = (const T*)h.cpsi[s];
  }
  return f;
}

template <typename T>
Fields<T> dev_fields(const fdtd_ctx* c) {
  Fields<T> f;
  f.Hx = (T*)field_ptr(c, 0);
  f.Hy = (T*)field_ptr(c, 1);
  f.Hz = (T*)field_ptr(c, 2);
  f.Ex = (T*)field_ptr(c, 3);
  f.Ey = (T*)field_ptr(c, 4);
  f.Ez = (T*)field_ptr(c, 5);
  return f;
}

template <typename T>
Sources<T> dev_sources(const fdtd_ctx* c) {
  Sources<T> s{};
  s.n = (int)c->src.size();
  for (int q = 0; q < s.n; q++) {
    s.box[q] = c->src[q].box;
    s.cs[q] = (const T*)c->src[q].cs;
    s.wave[q] = (const T*)c->src[q].wave;
  }
  return s;
}

Probes dev_probes(const fdtd_ctx* c) {
  Probes p{};
  p.n_v = (int)c->vprobe.size();
  p.n_i = (int)c->iprobe.size();
  for (int q = 0; q < p.n_v; q++) {
    p.v_comp[q] = c->vprobe[q].comp;
    p.v_count[q] = c->vprobe[q].count;
    p.v_idx[q] = c->vprobe[q].idx;
    p.v_csvf[q] = c->vprobe[q].csvf;
  }
  for (int q = 0; q < p.n_i; q++) {
    p.i_count[q] = c->iprobe[q].count;
    p.i_comp[q] = c->iprobe[q].comp;
    p.i_idx[q] = c->iprobe[q].idx;
    p.i_w[q] = c->iprobe[q].w;
  }
  p.V = c->V;
  p.I = c->I;
  p.nsteps = c->nsteps;
  p.status = c->d_status;
  return p;
}

FarField dev_ff(const fdtd_ctx* c) {
  FarField ff{};
  ff.nFreq = c->nFreq;
  if (c->nFreq == 0) return ff;
  ff.LI = c->li - 1; ff.LJ = c->lj - 1; ff.LK = c->lk - 1;
  ff.UI = c->ui - 1; ff.UJ = c->uj - 1; ff.UK = c->uk - 1;
  ff.ni = c->ui - c->li; ff.nj = c->uj - c->lj; ff.nk = c->uk - c->lk;
  ff.ph = c->ph;
  ff.acc = c->acc;
  for (int a = 0; a < 24; a++) ff.off[a] = c->ffoff[a];
  for (int a = 0; a < 3; a++) ff.sz[a] = c->ffsz[a];
  ff.kahan = c->acc_kahan;
  ff.block = c->dft_block;
  ff.samples = c->dft_samples;
  ff.done = c->d_dft_done;
  return ff;
}

// Trace buffers follow the probe counts.
int ensure_traces(fdtd_ctx* c) {
  const int nv = (int)c->vprobe.size(), ni = (int)c->iprobe.size();
  if (nv != c->nv_alloc) {
    dfree(c, c->V);
    c->V = nullptr;
    int rc = dalloc(c, (void**)&c->V, sizeof(double) * std::max(nv, 1) * (size_t)c->nsteps);
    if (rc) return rc;
    c->nv_alloc = nv;
  }
  if (ni != c->ni_alloc) {
    dfree(c, c->I);
    c->I = nullptr;
    int rc = dalloc(c, (void**)&c->I, sizeof(double) * std::max(ni, 1) * (size_t)c->nsteps);
    if (rc) return rc;
    c->ni_alloc = ni;
  }
  return FDTD_OK;
}

int check_ready(fdtd_ctx* c) {
  if (c->prec == FDTD_PREC_F32_TABLE) {
    for (int q = 0; q < 6; q++)
      if (!c->ids_set[q]) return fail(FDTD_ERR_STATE, "material ids of component %d not uploaded", q);
  } else {
    for (int q = 0; q < 18; q++)
      if (!c->coef_set[q]) return fail(FDTD_ERR_STATE, "coefficient array %d not uploaded", q);
  }
  return FDTD_OK;
}

// True when, on every axis, the two faces' H bands are disjoint and so are
// their E bands: a position then lies in at most one band per axis.
int bands_disjoint(const fdtd_ctx* c) {
  for (int a = 0; a < 3; a++) {
    const HostFace& n = c->face[2 * a];
    const HostFace& q = c->face[2 * a + 1];
    if (!n.present || !q.present || n.nc == 0 || q.nc == 0) continue;
    const bool h = n.m_start + n.nc <= q.m_start || q.m_start + q.nc <= n.m_start;
    const bool e = n.e_start + n.nc <= q.e_start || q.e_start + q.nc <= n.e_start;
    if (!h || !e) return 0;
  }
  return 1;
}

// Kernel parameters shared by both coefficient layouts.
template <typename T, class C>
StepParams<T, C> step_params(const fdtd_ctx* c, const C& coef) {
  StepParams<T, C> p{};
  p.g = GridDims{c->nx, c->ny, c->nz};
  p.f = dev_fields<T>(c);
  p.coef = coef;
  for (int q = 0; q < 6; q++) p.face[q] = dev_face<T>(c->face[q]);
  p.ex0b = (T*)c->ex0b;
  p.ts = c->d_ts;
  p.src = dev_sources<T>(c);
  p.dcell[0] = (T)c->dx;
  p.dcell[1] = (T)c->dy;
  p.dcell[2] = (T)c->dz;
  p.ichunk = c->ichunk;
  p.bands_disjoint = bands_disjoint(c);
  p.dft_block = c->dft_block;
  p.dft_done = c->d_dft_done;
  p.x_wall = c->x_wall;
  p.fault = c->d_status;
  return p;
}

// Step kernels for a prefetch depth: 1, 2 = planes prefetched in registers;
// 3, 4 = planes staged through shared memory (material-table problems only).
template <typename T, class C, bool EXACT>
void (*step_kernel(bool electric, int pf))(StepParams<T, C>) {
  if constexpr (C::kTable) {
    if (pf == 3) return electric ? k_step_e<T, C, EXACT, 3> : k_step_h<T, C, EXACT, 3>;
    if (pf == 4) return electric ? k_step_e<T, C, EXACT, 4> : k_step_h<T, C, EXACT, 4>;
    if (pf == 5) return electric ? k_step_e<T, C, EXACT, 5> : k_step_h<T, C, EXACT, 5>;
  }
  if (pf == 2) return electric ? k_step_e<T, C, EXACT, 2> : k_step_h<T, C, EXACT, 2>;
  return electric ? k_step_e<T, C, EXACT, 1> : k_step_h<T, C, EXACT, 1>;
}

// Dynamic shared memory of a step launch; raises the kernel's limit when the
// stages need more than the default 48 KB.
template <class K>
int stage_smem(K kernel, int pf, int threads, size_t* bytes) {
  *bytes = pf == 5 ? (size_t)bulk_smem_bytes(threads) : pf >= 3 ? (size_t)stage_smem_bytes(pf, threads) : 0;
  if (*bytes > 48 * 1024)
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*bytes));
  return FDTD_OK;
}

// Per-kernel timing of a profiled run: events around each launch.
struct KernelTimer {
  cudaEvent_t ev[5];
  double ms[4] = {0, 0, 0, 0};
};

// A launch shape is whole warps of at most 256 threads (the step kernels'
// launch bounds).
int check_block(int w, int rows) {
  const int t = w * rows;
  if ((w != 16 && w != 32) || t > 256 || t % 32 != 0)
    return fail(FDTD_ERR_BADARG, "block of %d x %d threads: need width 16 or 32, whole warps, at most 256", w, rows);
  return FDTD_OK;
}

// Enqueue `count` steps on stream `st` (default: the handle's stream; with
// `tm`, one step at a time, timing each kernel).
template <typename T, class C, bool EXACT>
int enqueue_steps(fdtd_ctx* c, const C& coef, int count, KernelTimer* tm = nullptr, cudaStream_t st = nullptr) {
  if (!st) st = c->stream;
  StepParams<T, C> p = step_params<T, C>(c, coef);
  Probes pr = dev_probes(c);
  FarField ff = dev_ff(c);
  // a thread per (j, k) column walks `ichunk` x planes
  int rc0 = check_block(c->block_w, c->block_rows);
  if (rc0) return rc0;
  if (c->prefetch == 5 && c->block_w != 32)
    return fail(FDTD_ERR_BADARG, "prefetch mode 5 (bulk-copied stages) needs 32-wide blocks, got %d", c->block_w);
  const dim3 blk(c->block_w, c->block_rows);
  const dim3 grd((c->nz + c->block_w) / c->block_w, (c->ny + c->block_rows) / c->block_rows,
                 (c->nx + 1 + c->ichunk - 1) / c->ichunk);
  const long long plane = (long long)c->ny * (c->nz + 1);
  const unsigned mid_blocks = (unsigned)((plane + pr.n_i + 255) / 256);
  const long long nff = (c->nFreq > 0) ? c->ffsz[0] + c->ffsz[1] + c->ffsz[2] : 0;
  const unsigned epi_blocks = (unsigned)((nff + pr.n_v + 255) / 256);
  const unsigned flush_blocks = (unsigned)((nff * std::max(c->nFreq, 1) + 255) / 256);
  auto kh = step_kernel<T, C, EXACT>(false, c->prefetch);
  auto ke = step_kernel<T, C, EXACT>(true, c->prefetch);
  size_t smem = 0;
  int rc = stage_smem(kh, c->prefetch, c->block_w * c->block_rows, &smem);
  if (!rc) rc = stage_smem(ke, c->prefetch, c->block_w * c->block_rows, &smem);
  if (rc) return rc;
  for (int s = 0; s < count; s++) {
    if (tm) CK(cudaEventRecord(tm->ev[0], st));
    kh<<<grd, blk, smem, st>>>(p);
    if (tm) CK(cudaEventRecord(tm->ev[1], st));
    k_step_mid<T, C, EXACT><<<mid_blocks, 256, 0, st>>>(p, pr);
    if (tm) CK(cudaEventRecord(tm->ev[2], st));
    ke<<<grd, blk, smem, st>>>(p);
    if (tm) CK(cudaEventRecord(tm->ev[3], st));
    if (epi_blocks) k_epilogue<T><<<epi_blocks, 256, 0, st>>>(p.f, p.g, ff, pr, c->d_ts);
    if (c->dft_block > 0) k_dft_flush<<<flush_blocks, 256, 0, st>>>(ff, c->d_ts, -1);
    if (tm) {
      CK(cudaEventRecord(tm->ev[4], st));
      CK(cudaEventSynchronize(tm->ev[4]));
      for (int q = 0; q < 4; q++) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, tm->ev[q], tm->ev[q + 1]));
        tm->ms[q] += ms;
      }
    }
  }
  CK(cudaGetLastError());
  return FDTD_OK;
}

template <typename T>
ArrayCoef<T> array_coef(const fdtd_ctx* c) {
  ArrayCoef<T> a{};
  for (int comp = 0; comp < 6; comp++)
    for (int w = 0; w < 3; w++) {
      const int id = comp < 3 ? 9 + 3 * comp + w : 3 * (comp - 3) + w;
      a.c[comp][w] = (const T*)c->coef[id];
    }
  return a;
}

// Material tables and 1/kappa profiles to the device (once per change; never
// called while the stream is being captured).
int prepare_table(fdtd_ctx* c, TableCoef* out) {
  const int n_axis[3] = {c->nx, c->ny, c->nz};
  if (!c->d_tab) {
    int rc = dalloc(c, (void**)&c->d_tab, 6 * kTableRows * 4 * sizeof(float));
    if (rc) return rc;
    for (int q = 0; q < 6; q++) {
      rc = dalloc(c, (void**)&c->d_invk[q], (n_axis[q % 3] + 1) * sizeof(float));
      if (rc) return rc;
    }
  }
  if (c->table_dirty) {
    std::vector<float> tab(6 * kTableRows * 4, 0.f);
    for (int f = 0; f < 6; f++) {
      const std::vector<float>& t = c->table[(f + 3) % 6];
      for (int r = 0; r < kTableRows; r++)
        for (int w = 0; w < 3; w++) tab[(f * kTableRows + r) * 4 + w] = t[3 * r + w];
    }
    CK(xfer(c, c->d_tab, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice));
    for (int a = 0; a < 3; a++) {
      std::vector<float> ie(n_axis[a] + 1, 1.f), im(n_axis[a] + 1, 1.f);
      for (int side = 0; side < 2; side++) {
        const HostFace& h = c->face[2 * a + side];
        if (!h.present) continue;
        std::vector<float> ke(h.nc), km(h.nc);
        CK(xfer(c, ke.data(), h.inv_k[0], h.nc * sizeof(float), cudaMemcpyDeviceToHost));
        CK(xfer(c, km.data(), h.inv_k[1], h.nc * sizeof(float), cudaMemcpyDeviceToHost));
        for (int q = 0; q < h.nc; q++) {
          ie[h.e_start + q] = ke[q];
          im[h.m_start + q] = km[q];
        }
      }
      CK(xfer(c, c->d_invk[a], ie.data(), ie.size() * sizeof(float), cudaMemcpyHostToDevice));
      CK(xfer(c, c->d_invk[3 + a], im.data(), im.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
  }
  TableCoef t{};
  for (int f = 0; f < 6; f++) t.ids[f] = c->ids[(f + 3) % 6];
  t.tab = (const float4*)c->d_tab;
  for (int q = 0; q < 6; q++) t.inv[q] = c->d_invk[q];
  *out = t;
  c->table_dirty = false;
  return FDTD_OK;
}

int enqueue(fdtd_ctx* c, int count, KernelTimer* tm = nullptr, cudaStream_t st = nullptr) {
  if (c->prec == FDTD_PREC_F64)
    return enqueue_steps<double, ArrayCoef<double>, true>(c, array_coef<double>(c), count, tm, st);
  if (c->prec == FDTD_PREC_F32)
    return enqueue_steps<float, ArrayCoef<float>, true>(c, array_coef<float>(c), count, tm, st);
  return enqueue_steps<float, TableCoef, false>(c, c->tcoef, count, tm, st);
}

// End of a run that reached step `upto` with the time-blocked DFT: accumulate
// what the run left buffered (the open block) and mark it done.
int close_dft_block(fdtd_ctx* c, int upto, cudaStream_t st) {
  if (c->dft_block <= 0) return FDTD_OK;
  if (upto % c->dft_block != 0) {
    const long long n = (c->ffsz[0] + c->ffsz[1] + c->ffsz[2]) * (long long)c->nFreq;
    k_dft_flush<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dev_ff(c), c->d_ts, upto);
    CK(cudaGetLastError());
  }
  CK(cudaMemcpyAsync(c->d_dft_done, &upto, sizeof(int), cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));  // `upto` is read from this frame
  return FDTD_OK;
}

constexpr int kGraphSteps = 64;       // shortest graph (and the cap's floor)
constexpr int kMaxGraphNodes = 40000;  // kernel launches held by one graph at most
constexpr size_t kMaxCachedGraphs = 6;

// The graph of `steps` steps from the cache, captured on `st` through `enq`
// (which enqueues that many steps) when missing.
template <class Enq>
int graph_for(RunGraphs& rg, cudaStream_t st, int steps, Enq enq, cudaGraphExec_t* out) {
  for (auto& e : rg.g)
    if (e.first == steps) {
      *out = e.second;
      return FDTD_OK;
    }
  if (rg.g.size() >= kMaxCachedGraphs) {
    cudaGraphExecDestroy(rg.g.front().second);
    rg.g.erase(rg.g.begin());
  }
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  int erc = enq(steps);
  cudaError_t ce = cudaStreamEndCapture(st, &g);
  if (erc) return erc;
  if (ce != cudaSuccess) return fail(FDTD_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
  cudaGraphExec_t ge = nullptr;
  ce = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return fail(FDTD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
  rg.g.push_back({steps, ge});
  *out = ge;
  return FDTD_OK;
}

// The graph launches of a run of `count` steps: full graphs of `cap` steps
// and one of the remainder, each captured (if missing) now.
template <class Enq>
int run_plan(RunGraphs& rg, cudaStream_t st, int count, int launches_per_step, Enq enq,
             std::vector<cudaGraphExec_t>* plan) {
  const int cap = std::max(kGraphSteps, kMaxGraphNodes / std::max(1, launches_per_step));
  plan->clear();
  if (count <= 0) return FDTD_OK;
  cudaGraphExec_t full = nullptr, rest = nullptr;
  if (count >= cap) {
    int rc = graph_for(rg, st, cap, enq, &full);
    if (rc) return rc;
  }
  if (count % cap) {
    int rc = graph_for(rg, st, count % cap, enq, &rest);
    if (rc) return rc;
  }
  for (int q = 0; q < count / cap; q++) plan->push_back(full);
  if (rest) plan->push_back(rest);
  return FDTD_OK;
}

constexpr int kMaxBatchStreams = 32;

int run_steps(fdtd_ctx* c, int count, float* elapsed_ms = nullptr, KernelTimer* tm = nullptr) {
  if (count < 0) return fail(FDTD_ERR_BADARG, "negative step count %d", count);
  if (c->ts + count > c->nsteps)
    return fail(FDTD_ERR_BADARG, "running %d steps from step %d exceeds numberOfTimeSteps=%d", count, c->ts,
                c->nsteps);
  int rc = check_ready(c);
  if (rc) return rc;
  rc = ensure_traces(c);
  if (rc) return rc;
  CK(cudaSetDevice(c->device));
  if (c->prec == FDTD_PREC_F32_TABLE && c->table_dirty) {
    rc = prepare_table(c, &c->tcoef);
    if (rc) return rc;
  }
  // the whole run as cached graphs, captured before the first launch
  if (c->dirty) {
    c->graphs.clear();
    c->dirty = false;
  }
  std::vector<cudaGraphExec_t> plan;
  if (!tm) {
    rc = run_plan(c->graphs, c->stream, count, c->dft_block > 0 ? 5 : 4,
                  [c](int n) { return enqueue(c, n); }, &plan);
    if (rc) return rc;
  }
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (elapsed_ms) {
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    CK(cudaEventRecord(ev0, c->stream));
  }
  if (tm) {
    rc = enqueue(c, count, tm);
    if (rc) return rc;
  }
  for (cudaGraphExec_t ge : plan) CK(cudaGraphLaunch(ge, c->stream));
  if (elapsed_ms) {
    CK(cudaEventRecord(ev1, c->stream));
    CK(cudaEventSynchronize(ev1));
    CK(cudaEventElapsedTime(elapsed_ms, ev0, ev1));
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
  }
  if (count > 0) {
    rc = close_dft_block(c, c->ts + count, c->stream);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(c->stream));
  c->ts += count;
  int st[2];
  CK(xfer(c, st, c->d_status, sizeof(st), cudaMemcpyDeviceToHost));
  if (st[0] == FDTD_ERR_CUDA) return fail(FDTD_ERR_CUDA, "a bounded device wait of the staged step ran out");
  if (st[0] != 0) return fail(FDTD_ERR_NONFINITE, "non-finite port sample at step %d", st[1]);
  return FDTD_OK;
}

unsigned long long mix64(unsigned long long h, unsigned long long w) {
  h ^= w;
  h *= 0xff51afd7ed558ccdULL;
  return h ^ (h >> 33);
}

// Folds `n` bytes at `p`, with the call's tag and the byte count, into the
// handle's set-up digest: eight independent lanes of eight bytes (so the
// multiplies overlap; a 168 MB material grid takes about 12 ms), then the
// remaining words and bytes.
void digest(fdtd_ctx* c, int tag, const void* p, size_t n) {
  unsigned long long h = mix64(c->setup_digest, ((unsigned long long)tag << 48) ^ (unsigned long long)n);
  const unsigned char* b = (const unsigned char*)p;
  size_t i = 0;
  if (n >= 64) {
    unsigned long long lane[8];
    for (int l = 0; l < 8; l++) lane[l] = h + 0x9e3779b97f4a7c15ULL * (unsigned long long)(l + 1);
    for (; i + 64 <= n; i += 64)
      for (int l = 0; l < 8; l++) {
        unsigned long long w;
        memcpy(&w, b + i + 8 * l, 8);
        lane[l] = mix64(lane[l], w);
      }
    for (int l = 0; l < 8; l++) h = mix64(h, lane[l]);
  }
  for (; i + 8 <= n; i += 8) {
    unsigned long long w;
    memcpy(&w, b + i, 8);
    h = mix64(h, w);
  }
  unsigned long long t = 0;
  for (; i < n; i++) t = (t << 8) | b[i];
  c->setup_digest = mix64(h, t);
}

void digest_vals(fdtd_ctx* c, int tag, std::initializer_list<double> v) {
  std::vector<double> a(v);
  digest(c, tag, a.data(), a.size() * sizeof(double));
}

}  // namespace

int fdtd_internal_traces(const fdtd_ctx* c, const double** V, const double** I, int* nsteps, int* steps,
                         int* device) {
  if (c->vprobe.empty() || c->iprobe.empty())
    return fail(FDTD_ERR_STATE, "handle has no voltage probe or no current probe");
  *V = c->V;
  *I = c->I;
  *nsteps = c->nsteps;
  *steps = c->ts;
  *device = c->device;
  return FDTD_OK;
}

// ===========================================================================
// Handle API
// ===========================================================================
extern "C" {

static int set_rows(fdtd_ctx* c, int comp, const std::vector<double>& rows);

const char* fdtd_last_error(void) { return g_err; }

int fdtd_device_count(int* count) {
  if (!count) return fail(FDTD_ERR_BADARG, "count is NULL");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
  *count = n;
  return FDTD_OK;
}

int fdtd_create(const FdtdConfig* cfg, fdtd_ctx** out) {
  if (!cfg || !out) return fail(FDTD_ERR_BADARG, "NULL argument");
  *out = nullptr;
  if (cfg->nx < 2 || cfg->ny < 2 || cfg->nz < 2) return fail(FDTD_ERR_BADARG, "grid %dx%dx%d too small", cfg->nx, cfg->ny, cfg->nz);
  if ((long long)(cfg->nx + 1) * (cfg->ny + 1) * (cfg->nz + 1) > (1LL << 31) - 1)
    return fail(FDTD_ERR_BADARG, "grid too large for 32-bit component indices");
  if (cfg->numberOfTimeSteps < 1) return fail(FDTD_ERR_BADARG, "numberOfTimeSteps must be >= 1");
  if (cfg->precision < FDTD_PREC_F64 || cfg->precision > FDTD_PREC_F32_TABLE)
    return fail(FDTD_ERR_BADARG, "unknown precision %d", cfg->precision);
  if (!(cfg->dx > 0 && cfg->dy > 0 && cfg->dz > 0 && cfg->dt > 0)) return fail(FDTD_ERR_BADARG, "non-positive spacing");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev)
    return fail(FDTD_ERR_CUDA, "CUDA device %d not available", cfg->device);
  fdtd_ctx* c = new fdtd_ctx();
  c->device = cfg->device;
  c->prec = cfg->precision;
  c->esz = (c->prec == FDTD_PREC_F64) ? 8 : 4;
  c->nx = cfg->nx; c->ny = cfg->ny; c->nz = cfg->nz;
  c->dx = cfg->dx; c->dy = cfg->dy; c->dz = cfg->dz; c->dt = cfg->dt;
  c->nsteps = cfg->numberOfTimeSteps;
  c->x_wall = c->prec == FDTD_PREC_F64 ? 0 : 1;
  digest_vals(c, 1, {(double)c->nx, (double)c->ny, (double)c->nz, c->dx, c->dy, c->dz, c->dt, (double)c->nsteps,
                     (double)c->prec});
  const long long nx = c->nx, ny = c->ny, nz = c->nz;
  c->ncomp[0] = (nx + 1) * ny * nz;
  c->ncomp[1] = nx * (ny + 1) * nz;
  c->ncomp[2] = nx * ny * (nz + 1);
  c->ncomp[3] = nx * (ny + 1) * (nz + 1);
  c->ncomp[4] = (nx + 1) * ny * (nz + 1);
  c->ncomp[5] = (nx + 1) * (ny + 1) * nz;
  int rc = FDTD_OK;
  if (cudaSetDevice(c->device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail(FDTD_ERR_CUDA, "cannot create a stream on device %d", cfg->device);
  }
  long long tot = 0;
  for (int q = 0; q < 6; q++) tot += c->ncomp[q];
  tot += (ny + 1) * (nz + 1) + 64;  // slack plane past Ez
  if (!rc) rc = dalloc(c, &c->fields, tot * c->esz);
  if (!rc) rc = dalloc(c, &c->ex0b, (size_t)(ny + 1) * (nz + 1) * c->esz);
  if (!rc) rc = dalloc(c, (void**)&c->d_ts, sizeof(int));
  if (!rc) rc = dalloc(c, (void**)&c->d_status, 2 * sizeof(int));
  if (!rc) {
    int init_ts = -1;
    int st[2] = {0, 1 << 30};
    if (xfer(c, c->d_ts, &init_ts, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        xfer(c, c->d_status, st, sizeof(st), cudaMemcpyHostToDevice) != cudaSuccess)
      rc = fail(FDTD_ERR_CUDA, "cannot initialise step counter");
  }
  if (!rc && c->prec != FDTD_PREC_F32_TABLE) {
    for (int q = 0; q < 18 && !rc; q++) rc = dalloc(c, &c->coef[q], coef_count(c, q) * c->esz);
  }
  if (!rc && c->prec == FDTD_PREC_F32_TABLE) {
    // 64 bytes of padding: the staged kernels copy whole aligned words of ids,
    // and the bulk-copied rows (32 ids widened to 16-byte boundaries) may
    // reach up to 47 bytes past the last id
    for (int q = 0; q < 6 && !rc; q++) rc = dalloc(c, (void**)&c->ids[q], c->ncomp[(q + 3) % 6] + 64);
  }
  if (!rc) rc = ensure_traces(c);
  if (!rc) {
    // default launch shape: enough x chunks for about four waves of 2048-thread SMs
    const long long cols = (long long)(ny + 1) * (nz + 1);
    const long long want = 4LL * 148 * 2048;
    long long ch = cols * (nx + 1) / want;
    c->ichunk = (int)std::max<long long>(1, std::min<long long>(64, ch));
  }
  if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = fail(FDTD_ERR_CUDA, "stream sync failed");
  if (rc) {
    std::string msg = g_err;
    fdtd_free(c);
    return fail(rc, "%s", msg.c_str());
  }
  *out = c;
  return FDTD_OK;
}

void fdtd_free(fdtd_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->graphs.clear();
  for (void* p : c->owned) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int fdtd_ctx_upload_coeff(fdtd_ctx* c, int which, const double* host, long n) {
  if (!c || !host) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (c->prec == FDTD_PREC_F32_TABLE) return fail(FDTD_ERR_STATE, "material-table problem takes fdtd_ctx_upload_material");
  if (which < 0 || which >= 18) return fail(FDTD_ERR_BADARG, "coefficient id %d out of range 0..17", which);
  if (n != coef_count(c, which)) return fail(FDTD_ERR_BADARG, "coefficient %d: got %ld values, expected %lld", which, n, coef_count(c, which));
  digest_vals(c, 2, {(double)which});
  digest(c, 2, host, (size_t)n * sizeof(double));
  CK(cudaSetDevice(c->device));
  int rc = upload_real(c, c->coef[which], host, n);
  if (!rc) c->coef_set[which] = true;
  c->coef_device = false;  // host arrays carry their own kappa division and come with CPsi
  return rc;
}

// The CPML bands of face f on the four per-cell FP64 coefficient arrays its
// Psi slots correct (cpml.js:212-243): per slot, CPsi = coefficient x cell size
// over the band (into the face's CPsi array), then the coefficient is divided
// by kappa of its band cell.  Slots: x face Chyez Chzey Ceyhz Cezhy, y face
// Chxez Chzex Cezhx Cexhz, z face Chxey Chyex Cexhy Ceyhx (ids as in
// fdtd_ctx_upload_coeff); the H slots use the H band and kappa_m, the E slots
// the E band and kappa_e.
static int cpml_band_on_device(fdtd_ctx* c, int f, const double* kappa_e, const double* kappa_m) {
  static const int coef_id[3][4] = {{13, 17, 5, 7}, {11, 16, 8, 1}, {10, 14, 2, 4}};
  const int axis = f / 2;
  HostFace& h = c->face[f];
  const double cell = axis == 0 ? c->dx : (axis == 1 ? c->dy : c->dz);
  double* d_kap = nullptr;
  if (cudaMalloc((void**)&d_kap, 2 * h.nc * sizeof(double)) != cudaSuccess) return fail(FDTD_ERR_OOM, "kappa profiles");
  int rc = FDTD_OK;
  if (xfer(c, d_kap, kappa_e, h.nc * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      xfer(c, d_kap + h.nc, kappa_m, h.nc * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = fail(FDTD_ERR_CUDA, "kappa upload");
  for (int s = 0; s < 4 && !rc; s++) {
    const int id = coef_id[axis][s], comp = id / 3;   // API order Ex Ey Ez Hx Hy Hz
    const int ni = (comp == 0 || comp == 4 || comp == 5) ? c->nx : c->nx + 1;
    const int nj = (comp == 1 || comp == 3 || comp == 5) ? c->ny : c->ny + 1;
    const int nk = (comp == 2 || comp == 3 || comp == 4) ? c->nz : c->nz + 1;
    const int st = s < 2 ? h.m_start : h.e_start;
    const long long n = (long long)(axis == 0 ? h.nc : ni) * (axis == 1 ? h.nc : nj) * (axis == 2 ? h.nc : nk);
    if (n != h.n[s]) { rc = fail(FDTD_ERR_STATE, "face %d slot %d: band of %lld cells, Psi of %lld", f, s, n, h.n[s]); break; }
    k_cpml_band<<<148 * 8, 256, 0, c->stream>>>((double*)c->coef[id], ni, nj, nk, axis, st, h.nc, cell,
                                                s < 2 ? d_kap + h.nc : d_kap, (double*)h.cpsi[s]);
  }
  if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess)
    rc = fail(FDTD_ERR_CUDA, "CPML band: %s", cudaGetErrorString(cudaGetLastError()));
  cudaFree(d_kap);
  if (!rc) c->kappa_done[f] = true;
  return rc;
}

int fdtd_ctx_upload_cpml(fdtd_ctx* c, int f, int nc, const double* b_e, const double* a_e, const double* b_m,
                         const double* a_m, const double* kappa_e, const double* kappa_m, const double* CPsi0,
                         long n0, const double* CPsi1, long n1, const double* CPsi2, long n2, const double* CPsi3,
                         long n3, int m_start, int e_start) {
  if (!c) return fail(FDTD_ERR_BADARG, "NULL handle");
  if (f < 0 || f >= 6) return fail(FDTD_ERR_BADARG, "face id %d out of range 0..5", f);
  if (nc < 0) return fail(FDTD_ERR_BADARG, "negative cell count");
  const int axis_n = f / 2 == 0 ? c->nx : (f / 2 == 1 ? c->ny : c->nz);
  if (nc > axis_n / 2) return fail(FDTD_ERR_BADARG, "face %d: %d CPML cells do not fit in %d cells", f, nc, axis_n);
  if (m_start < 0 || m_start + nc > axis_n) return fail(FDTD_ERR_BADARG, "face %d: H band [%d,%d) outside [0,%d)", f, m_start, m_start + nc, axis_n);
  if (e_start < 1 || e_start + nc > axis_n) return fail(FDTD_ERR_BADARG, "face %d: E band [%d,%d) outside [1,%d)", f, e_start, e_start + nc, axis_n);
  if (nc > 0 && (!b_e || !a_e || !b_m || !a_m)) return fail(FDTD_ERR_BADARG, "face %d: missing b/a profile", f);
  const bool table = c->prec == FDTD_PREC_F32_TABLE;
  if (table && nc > 0 && (!kappa_e || !kappa_m)) return fail(FDTD_ERR_BADARG, "face %d: material-table problems need kappa profiles", f);
  long long want[4];
  psi_sizes(c, f, nc, want);
  const double* cp[4] = {CPsi0, CPsi1, CPsi2, CPsi3};
  const long got[4] = {n0, n1, n2, n3};
  digest_vals(c, 3, {(double)f, (double)nc, (double)m_start, (double)e_start, (double)n0, (double)n1, (double)n2,
                     (double)n3});
  for (const double* prof : {b_e, a_e, b_m, a_m, kappa_e, kappa_m})
    if (prof && nc > 0) digest(c, 3, prof, (size_t)nc * sizeof(double));
  for (int s = 0; s < 4; s++)
    if (cp[s] && got[s] > 0) digest(c, 3, cp[s], (size_t)got[s] * sizeof(double));
  // FP64 coefficients built on the device and no CPsi given: CPsi and the
  // kappa division of the band are done here, on the device
  const bool dev = !table && c->coef_device && !CPsi0 && !CPsi1 && !CPsi2 && !CPsi3 && !n0 && !n1 && !n2 && !n3;
  if (dev && nc > 0) {
    if (!kappa_e || !kappa_m) return fail(FDTD_ERR_BADARG, "face %d: device-built coefficients need kappa profiles", f);
    if (c->kappa_done[f]) return fail(FDTD_ERR_STATE, "face %d: its band was already divided by kappa; rebuild the coefficients first", f);
    for (int q = 0; q < nc; q++)
      if (!(kappa_e[q] > 0) || !(kappa_m[q] > 0)) return fail(FDTD_ERR_BADARG, "face %d: kappa must be positive", f);
  }
  for (int s = 0; s < 4; s++) {
    if (table || dev) continue;  // CPsi comes from the coefficient tables, or is made on the device
    if (got[s] != want[s] || (want[s] > 0 && !cp[s]))
      return fail(FDTD_ERR_BADARG, "face %d slot %d: got %ld CPsi values, expected %lld", f, s, got[s], want[s]);
  }
  CK(cudaSetDevice(c->device));
  HostFace& h = c->face[f];
  for (int s = 0; s < 4; s++) { dfree(c, h.prof[s]); dfree(c, h.psi[s]); dfree(c, h.cpsi[s]); }
  dfree(c, h.inv_k[0]); dfree(c, h.inv_k[1]);
  h = HostFace();
  h.present = nc > 0;
  h.nc = nc; h.m_start = m_start; h.e_start = e_start;
  invalidate(c);
  if (nc == 0) return FDTD_OK;
  const double* pr[4] = {b_e, a_e, b_m, a_m};
  int rc = FDTD_OK;
  for (int s = 0; s < 4 && !rc; s++) {
    rc = dalloc(c, &h.prof[s], nc * c->esz);
    if (!rc) rc = upload_real(c, h.prof[s], pr[s], nc);
  }
  for (int s = 0; s < 4 && !rc; s++) {
    h.n[s] = want[s];
    rc = dalloc(c, &h.psi[s], want[s] * c->esz);
    if (!rc && !table) {
      rc = dalloc(c, &h.cpsi[s], want[s] * c->esz);
      if (!rc && !dev) rc = upload_real(c, h.cpsi[s], cp[s], want[s]);
    }
  }
  if (!rc && dev) rc = cpml_band_on_device(c, f, kappa_e, kappa_m);
  if (!rc && table) {
    std::vector<float> ik(nc);
    const double* kp[2] = {kappa_e, kappa_m};
    for (int s = 0; s < 2 && !rc; s++) {
      for (int q = 0; q < nc; q++) {
        if (!(kp[s][q] > 0)) return fail(FDTD_ERR_BADARG, "face %d: kappa must be positive", f);
        ik[q] = (float)(1.0 / kp[s][q]);
      }
      rc = dalloc(c, (void**)&h.inv_k[s], nc * sizeof(float));
      if (!rc && xfer(c, h.inv_k[s], ik.data(), nc * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = fail(FDTD_ERR_CUDA, "kappa upload failed");
    }
  }
  if (rc) h.present = false;
  return rc;
}

int fdtd_ctx_add_vsource(fdtd_ctx* c, int dir, const int* idx, const double* coef, int count, const double* wave,
                         int nSteps) {
  if (!c || !idx || !coef || !wave) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (dir < 0 || dir > 2) return fail(FDTD_ERR_BADARG, "source direction %d not in 0..2", dir);
  if (count <= 0) return fail(FDTD_ERR_BADARG, "source has no cells");
  if (nSteps < c->nsteps) return fail(FDTD_ERR_BADARG, "waveform has %d values, need %d", nSteps, c->nsteps);
  if ((int)c->src.size() >= kMaxSources) return fail(FDTD_ERR_BADARG, "at most %d sources", kMaxSources);
  digest_vals(c, 4, {(double)dir, (double)count});
  digest(c, 4, idx, (size_t)count * sizeof(int));
  digest(c, 4, coef, (size_t)count * sizeof(double));
  digest(c, 4, wave, (size_t)c->nsteps * sizeof(double));
  // component extents of E_dir
  const int ni = dir == 0 ? c->nx : c->nx + 1, nj = dir == 1 ? c->ny : c->ny + 1, nk = dir == 2 ? c->nz : c->nz + 1;
  const long long n = (long long)ni * nj * nk;
  int bi0 = 1 << 30, bi1 = -1, bj0 = 1 << 30, bj1 = -1, bk0 = 1 << 30, bk1 = -1;
  for (int q = 0; q < count; q++) {
    if (idx[q] < 0 || idx[q] >= n) return fail(FDTD_ERR_BADARG, "source index %d out of range", idx[q]);
    const int i = idx[q] / (nj * nk), j = (idx[q] / nk) % nj, k = idx[q] % nk;
    bi0 = std::min(bi0, i); bi1 = std::max(bi1, i);
    bj0 = std::min(bj0, j); bj1 = std::max(bj1, j);
    bk0 = std::min(bk0, k); bk1 = std::max(bk1, k);
  }
  // the list must be the box in createLinearIndexList order (grid.js:228-243)
  const long long bn = (long long)(bi1 - bi0 + 1) * (bj1 - bj0 + 1) * (bk1 - bk0 + 1);
  if (bn != count) return fail(FDTD_ERR_BADARG, "source cells do not form a box");
  int q = 0;
  for (int k = bk0; k <= bk1; k++)
    for (int j = bj0; j <= bj1; j++)
      for (int i = bi0; i <= bi1; i++, q++)
        if (idx[q] != (i * nj + j) * nk + k) return fail(FDTD_ERR_BADARG, "source cells not in k-j-i box order");
  for (int q2 = 0; q2 < count; q2++)
    if (!std::isfinite(coef[q2])) return fail(FDTD_ERR_BADARG, "non-finite source coefficient");
  CK(cudaSetDevice(c->device));
  HostSource s;
  s.box = SourceBox{dir, bi0, bi1, bj0, bj1, bk0, bk1};
  s.count = count;
  int rc = dalloc(c, &s.cs, count * c->esz);
  if (!rc) rc = upload_real(c, s.cs, coef, count);
  if (!rc) rc = dalloc(c, &s.wave, (size_t)c->nsteps * c->esz);
  if (!rc) rc = upload_real(c, s.wave, wave, c->nsteps);
  if (rc) return rc;
  c->src.push_back(s);
  invalidate(c);
  return FDTD_OK;
}

int fdtd_ctx_add_svoltage(fdtd_ctx* c, int dir, const int* idx, int count, double Csvf) {
  if (!c || !idx) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (dir < 0 || dir > 2) return fail(FDTD_ERR_BADARG, "probe direction %d not in 0..2", dir);
  if (count <= 0) return fail(FDTD_ERR_BADARG, "probe has no cells");
  if ((int)c->vprobe.size() >= kMaxProbes) return fail(FDTD_ERR_BADARG, "at most %d voltage probes", kMaxProbes);
  const long long n = c->ncomp[3 + dir];
  for (int q = 0; q < count; q++)
    if (idx[q] < 0 || idx[q] >= n) return fail(FDTD_ERR_BADARG, "probe index %d out of range", idx[q]);
  digest_vals(c, 5, {(double)dir, (double)count, Csvf});
  digest(c, 5, idx, (size_t)count * sizeof(int));
  CK(cudaSetDevice(c->device));
  HostVProbe p{dir, count, nullptr, Csvf};
  int rc = dalloc(c, (void**)&p.idx, count * sizeof(int));
  if (rc) return rc;
  CK(xfer(c, p.idx, idx, count * sizeof(int), cudaMemcpyHostToDevice));
  c->vprobe.push_back(p);
  invalidate(c);
  return ensure_traces(c);
}

int fdtd_ctx_add_scurrent(fdtd_ctx* c, const int* comp, const int* idx, const double* w, int count) {
  if (!c || !comp || !idx || !w) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (count <= 0) return fail(FDTD_ERR_BADARG, "probe has no samples");
  if ((int)c->iprobe.size() >= kMaxProbes) return fail(FDTD_ERR_BADARG, "at most %d current probes", kMaxProbes);
  for (int q = 0; q < count; q++) {
    if (comp[q] < 0 || comp[q] > 2) return fail(FDTD_ERR_BADARG, "current probe component %d not in 0..2", comp[q]);
    if (idx[q] < 0 || idx[q] >= c->ncomp[comp[q]]) return fail(FDTD_ERR_BADARG, "current probe index %d out of range", idx[q]);
  }
  digest_vals(c, 6, {(double)count});
  digest(c, 6, comp, (size_t)count * sizeof(int));
  digest(c, 6, idx, (size_t)count * sizeof(int));
  digest(c, 6, w, (size_t)count * sizeof(double));
  CK(cudaSetDevice(c->device));
  HostIProbe p{count, nullptr, nullptr, nullptr};
  int rc = dalloc(c, (void**)&p.comp, count * sizeof(int));
  if (!rc) rc = dalloc(c, (void**)&p.idx, count * sizeof(int));
  if (!rc) rc = dalloc(c, (void**)&p.w, count * sizeof(double));
  if (rc) return rc;
  CK(xfer(c, p.comp, comp, count * sizeof(int), cudaMemcpyHostToDevice));
  CK(xfer(c, p.idx, idx, count * sizeof(int), cudaMemcpyHostToDevice));
  CK(xfer(c, p.w, w, count * sizeof(double), cudaMemcpyHostToDevice));
  c->iprobe.push_back(p);
  invalidate(c);
  return ensure_traces(c);
}

int fdtd_ctx_setup_farfield(fdtd_ctx* c, int nFreq, const double* freqs, int li, int lj, int lk, int ui, int uj,
                            int uk) {
  if (!c) return fail(FDTD_ERR_BADARG, "NULL handle");
  if (nFreq < 0 || (nFreq > 0 && !freqs)) return fail(FDTD_ERR_BADARG, "bad frequency list");
  if (c->nFreq > 0) return fail(FDTD_ERR_STATE, "far field already set up");
  if (nFreq == 0) return FDTD_OK;
  // the 4-point averages reach one cell outside the box on each side
  if (li < 2 || lj < 2 || lk < 2 || ui > c->nx || uj > c->ny || uk > c->nz || ui <= li || uj <= lj || uk <= lk)
    return fail(FDTD_ERR_BADARG, "Huygens box [%d,%d]x[%d,%d]x[%d,%d] does not fit the grid", li, ui, lj, uj, lk, uk);
  digest_vals(c, 7, {(double)nFreq, (double)li, (double)lj, (double)lk, (double)ui, (double)uj, (double)uk});
  digest(c, 7, freqs, (size_t)nFreq * sizeof(double));
  CK(cudaSetDevice(c->device));
  c->nFreq = nFreq;
  c->ffreq.assign(freqs, freqs + nFreq);
  c->li = li; c->lj = lj; c->lk = lk; c->ui = ui; c->uj = uj; c->uk = uk;
  const long long ni = ui - li, nj = uj - lj, nk = uk - lk;
  c->ffsz[0] = nj * nk;
  c->ffsz[1] = ni * nk;
  c->ffsz[2] = ni * nj;
  long long off = 0;
  for (int a = 0; a < 24; a++) {
    c->ffoff[a] = off;
    off += 2 * nFreq * c->ffsz[(a % 12) / 4];
  }
  int rc = dalloc(c, (void**)&c->acc, off * sizeof(double));
  if (rc) return rc;
  // phasors, evaluated as farfield.js:101-110 does
  std::vector<double> ph((size_t)c->nsteps * nFreq * 4);
  for (int ts = 0; ts < c->nsteps; ts++)
    for (int m = 0; m < nFreq; m++) {
      const double w = 2 * M_PI * freqs[m];
      const double wdt = w * c->dt;
      const double phh = wdt * (ts + 0.5), phe = wdt * (ts + 1);
      double* q = &ph[((size_t)ts * nFreq + m) * 4];
      q[0] = std::cos(phh);
      q[1] = -std::sin(phh);
      q[2] = std::cos(phe);
      q[3] = -std::sin(phe);
    }
  rc = dalloc(c, (void**)&c->ph, ph.size() * sizeof(double));
  if (rc) return rc;
  CK(xfer(c, c->ph, ph.data(), ph.size() * sizeof(double), cudaMemcpyHostToDevice));
  invalidate(c);
  return FDTD_OK;
}

int fdtd_ctx_upload_material(fdtd_ctx* c, int comp, const unsigned char* ids, long n, const double* table, int rows) {
  if (!c || !ids || !table) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (c->prec != FDTD_PREC_F32_TABLE) return fail(FDTD_ERR_STATE, "not a material-table problem");
  if (comp < 0 || comp > 5) return fail(FDTD_ERR_BADARG, "component %d not in 0..5", comp);
  const long long want = c->ncomp[(comp + 3) % 6];
  if (n != want) return fail(FDTD_ERR_BADARG, "component %d: got %ld ids, expected %lld", comp, n, want);
  if (rows < 1 || rows > kTableRows) return fail(FDTD_ERR_BADARG, "table rows %d not in 1..%d", rows, kTableRows);
  for (long q = 0; q < n; q++)
    if (ids[q] >= rows) return fail(FDTD_ERR_BADARG, "material id %d >= table rows %d", ids[q], rows);
  digest_vals(c, 8, {(double)comp, (double)rows});
  digest(c, 8, ids, (size_t)n);
  digest(c, 8, table, (size_t)rows * 3 * sizeof(double));
  CK(cudaSetDevice(c->device));
  CK(xfer(c, c->ids[comp], ids, n, cudaMemcpyHostToDevice));
  int rc = set_rows(c, comp, std::vector<double>(table, table + 3 * rows));
  if (rc) return rc;
  c->ids_set[comp] = true;
  invalidate(c);
  return FDTD_OK;
}

// Coefficient triple (self, curl1, curl2) of a component for an averaged
// material pair, as coefficients.js:22-116 evaluates it (no kappa).
static void coef_row(const fdtd_ctx* c, int comp, double e, double s, double out[3]) {
  const double dt = c->dt;
  const double tdx = 2 * dt / c->dx, tdy = 2 * dt / c->dy, tdz = 2 * dt / c->dz;
  const double scale = comp < 3 ? 8.854187817e-12 : 4 * M_PI * 1e-7;
  const double a = 2 * e * scale;
  const double b = dt * s;
  const double denom = a + b;
  // curl numerators (coefficients.js:32-106): Ex tdy,-tdz | Ey tdz,-tdx | Ez tdx,-tdy |
  // Hx tdz,-tdy | Hy tdx,-tdz | Hz tdy,-tdx
  static const int sel1[6] = {1, 2, 0, 2, 0, 1}, sel2[6] = {2, 0, 1, 1, 2, 0};
  const double t[3] = {tdx, tdy, tdz};
  const double n1 = t[sel1[comp]];
  const double n2 = -t[sel2[comp]];
  out[0] = (a - b) / denom;
  out[1] = n1 / denom;
  out[2] = n2 / denom;
}

static int set_rows(fdtd_ctx* c, int comp, const std::vector<double>& rows) {
  const int nrows = (int)rows.size() / 3;
  if (nrows > kTableRows) return fail(FDTD_ERR_BADARG, "component %d needs %d coefficient rows (limit %d)", comp, nrows, kTableRows);
  c->rows64[comp] = rows;
  c->table[comp].assign(3 * kTableRows, 0.f);
  for (size_t r = 0; r < rows.size(); r++) c->table[comp][r] = (float)rows[r];
  return FDTD_OK;
}

int fdtd_ctx_build_material(fdtd_ctx* c, const unsigned char* mat, long ncells, int ntypes, const double* props,
                            int nplates, const int* plates, const double* plate_sigma) {
  if (!c || !mat || !props || (nplates > 0 && (!plates || !plate_sigma))) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (c->prec == FDTD_PREC_F32)
    return fail(FDTD_ERR_STATE, "per-cell FP32 problems take fdtd_ctx_upload_coeff (FP64 and material-table problems build here)");
  const bool f64 = c->prec == FDTD_PREC_F64;
  if (ncells != (long)c->nx * c->ny * c->nz) return fail(FDTD_ERR_BADARG, "material grid of %ld cells, need %lld", ncells, (long long)c->nx * c->ny * c->nz);
  if (ntypes < 1 || ntypes > 48) return fail(FDTD_ERR_BADARG, "%d material slots (1..48 supported)", ntypes);
  if (nplates < 0 || nplates > kMaxPlates) return fail(FDTD_ERR_BADARG, "%d plates (at most %d)", nplates, kMaxPlates);
  unsigned char mmax = 0;
  for (long q = 0; q < ncells; q++) mmax = std::max(mmax, mat[q]);
  if (mmax >= ntypes) return fail(FDTD_ERR_BADARG, "material id %d has no properties", mmax);
  digest_vals(c, 9, {(double)ncells, (double)ntypes, (double)nplates});
  digest(c, 9, mat, (size_t)ncells);
  digest(c, 9, props, (size_t)ntypes * 4 * sizeof(double));
  if (nplates > 0) {
    digest(c, 9, plates, (size_t)nplates * 7 * sizeof(int));
    digest(c, 9, plate_sigma, (size_t)nplates * sizeof(double));
  }
  MatBuild b{};
  b.nx = c->nx; b.ny = c->ny; b.nz = c->nz; b.M = ntypes; b.nplates = nplates;
  std::vector<double> psig;  // distinct plate conductivities
  const int ext[3][3] = {{c->nx, c->ny + 1, c->nz + 1}, {c->nx + 1, c->ny, c->nz + 1}, {c->nx + 1, c->ny + 1, c->nz}};
  for (int q = 0; q < nplates; q++) {
    const int* P = plates + 7 * q;
    if (P[0] < 0 || P[0] > 2) return fail(FDTD_ERR_BADARG, "plate %d: component %d not in 0..2", q, P[0]);
    const int* e = ext[P[0]];
    if (P[1] < 0 || P[2] >= e[0] || P[3] < 0 || P[4] >= e[1] || P[5] < 0 || P[6] >= e[2] || P[1] > P[2] || P[3] > P[4] || P[5] > P[6])
      return fail(FDTD_ERR_BADARG, "plate %d: box outside its component array", q);
    int sid = -1;
    for (size_t u = 0; u < psig.size(); u++)
      if (psig[u] == plate_sigma[q]) sid = (int)u;
    if (sid < 0) { sid = (int)psig.size(); psig.push_back(plate_sigma[q]); }
    b.plate[q] = PlateBox{P[0], P[1], P[2], P[3], P[4], P[5], P[6], sid};
  }
  CK(cudaSetDevice(c->device));
  unsigned char* d_mat = nullptr;
  uint8_t *d_present = nullptr, *d_map = nullptr;
  int* d_map64 = nullptr;     // FP64: code -> row
  double* d_rows = nullptr;   // FP64: row triples
  const long long M = ntypes;
  const long long ncode_e = (M * M * M * M + 1) * (long long)(psig.size() + 1);
  const long long ncode_h = M * M + 1;
  int rc = FDTD_OK;
  if (cudaMalloc(&d_mat, ncells) != cudaSuccess || cudaMalloc(&d_present, std::max(ncode_e, ncode_h)) != cudaSuccess ||
      cudaMalloc(&d_map, std::max(ncode_e, ncode_h)) != cudaSuccess ||
      (f64 && cudaMalloc((void**)&d_map64, std::max(ncode_e, ncode_h) * sizeof(int)) != cudaSuccess)) {
    rc = fail(FDTD_ERR_OOM, "material build buffers");
  }
  if (!rc && xfer(c, d_mat, mat, ncells, cudaMemcpyHostToDevice) != cudaSuccess) rc = fail(FDTD_ERR_CUDA, "material grid upload");
  b.mat = d_mat;
  const double* t_eps = props;  // props rows: eps_r, mu_r, sigma_e, sigma_m per type id
  std::vector<uint8_t> present, map;
  for (int comp = 0; comp < 6 && !rc; comp++) {
    const long long ncode = comp < 3 ? ncode_e : ncode_h;
    present.assign(ncode, 0);
    if (cudaMemsetAsync(d_present, 0, ncode, c->stream) != cudaSuccess) { rc = fail(FDTD_ERR_CUDA, "memset"); break; }
    k_material_mark<<<148 * 8, 256, 0, c->stream>>>(b, comp, d_present);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess ||
        xfer(c, present.data(), d_present, ncode, cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = fail(FDTD_ERR_CUDA, "material mark: %s", cudaGetErrorString(cudaGetLastError()));
      break;
    }
    std::map<std::pair<double, double>, int> rowof;
    std::vector<double> rows;
    std::vector<int> row_of_code(f64 ? ncode : 0, 0);
    map.assign(ncode, 0);
    const long long fill = comp < 3 ? M * M * M * M : M * M;
    for (long long code = 0; code < ncode; code++) {
      if (!present[code]) continue;
      double e, s;
      if (comp < 3) {
        const long long base = code % (fill + 1), sid = code / (fill + 1) - 1;
        if (base == fill) {
          e = 1.0; s = 0.0;
        } else {
          const long long m1 = base % M, m2 = (base / M) % M, m3 = (base / (M * M)) % M, m4 = base / (M * M * M);
          e = 0.25 * (t_eps[4 * m1] + t_eps[4 * m2] + t_eps[4 * m3] + t_eps[4 * m4]);
          s = 0.25 * (props[4 * m1 + 2] + props[4 * m2 + 2] + props[4 * m3 + 2] + props[4 * m4 + 2]);
        }
        if (sid >= 0) s = psig[sid];
      } else if (code == fill) {
        e = 1.0; s = 0.0;
      } else {
        const long long m1 = code % M, m2 = code / M;
        const double mu1 = props[4 * m1 + 1], mu2 = props[4 * m2 + 1];
        e = 2 * mu1 * mu2 / (mu1 + mu2);
        const double sm1 = props[4 * m1 + 3], sm2 = props[4 * m2 + 3];
        s = 2 * sm1 * sm2 / (sm1 + sm2);
      }
      auto key = std::make_pair(e, s);
      auto it = rowof.find(key);
      int r;
      if (it == rowof.end()) {
        r = (int)rows.size() / 3;
        rowof[key] = r;
        double tr[3];
        coef_row(c, comp, e, s, tr);
        rows.insert(rows.end(), tr, tr + 3);
      } else {
        r = it->second;
      }
      map[code] = (uint8_t)std::min(r, 255);
      if (f64) row_of_code[code] = r;
    }
    if (f64) {
      // every cell takes its row's FP64 triple: coefficient arrays 3 comp .. 3 comp + 2
      const std::vector<int>& map64 = row_of_code;
      cudaFree(d_rows);
      d_rows = nullptr;
      if (cudaMalloc((void**)&d_rows, std::max<size_t>(rows.size(), 1) * sizeof(double)) != cudaSuccess) {
        rc = fail(FDTD_ERR_OOM, "coefficient rows");
        break;
      }
      if (xfer(c, d_rows, rows.data(), rows.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
          xfer(c, d_map64, map64.data(), ncode * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = fail(FDTD_ERR_CUDA, "coefficient row upload");
        break;
      }
      k_material_coef<<<148 * 8, 256, 0, c->stream>>>(b, comp, d_map64, d_rows, (double*)c->coef[3 * comp],
                                                      (double*)c->coef[3 * comp + 1], (double*)c->coef[3 * comp + 2]);
      if (cudaStreamSynchronize(c->stream) != cudaSuccess) { rc = fail(FDTD_ERR_CUDA, "coefficients: %s", cudaGetErrorString(cudaGetLastError())); break; }
      for (int w = 0; w < 3; w++) c->coef_set[3 * comp + w] = true;
      continue;
    }
    rc = set_rows(c, comp, rows);
    if (rc) break;
    if (xfer(c, d_map, map.data(), ncode, cudaMemcpyHostToDevice) != cudaSuccess) { rc = fail(FDTD_ERR_CUDA, "code map upload"); break; }
    k_material_ids<<<148 * 8, 256, 0, c->stream>>>(b, comp, d_map, c->ids[comp]);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) { rc = fail(FDTD_ERR_CUDA, "material ids: %s", cudaGetErrorString(cudaGetLastError())); break; }
    c->ids_set[comp] = true;
  }
  cudaFree(d_mat);
  cudaFree(d_present);
  cudaFree(d_map);
  cudaFree(d_map64);
  cudaFree(d_rows);
  if (f64) {
    c->coef_device = rc == FDTD_OK;
    for (int f = 0; f < 6; f++) c->kappa_done[f] = false;
  }
  invalidate(c);
  return rc;
}

// FP64 problems: the triples overwrite coefficient arrays 3 comp .. 3 comp + 2 at the cells.
static int override_coef64(fdtd_ctx* c, int comp, const int* idx, const double* triples, int count) {
  if (comp < 0 || comp > 5) return fail(FDTD_ERR_BADARG, "component %d not in 0..5", comp);
  for (int w = 0; w < 3; w++)
    if (!c->coef_set[3 * comp + w]) return fail(FDTD_ERR_STATE, "component %d has no coefficients yet", comp);
  if (count <= 0) return FDTD_OK;
  const long long n = coef_count(c, 3 * comp);
  for (int q = 0; q < count; q++) {
    if (idx[q] < 0 || idx[q] >= n) return fail(FDTD_ERR_BADARG, "cell index %d out of range", idx[q]);
    for (int w = 0; w < 3; w++)
      if (!std::isfinite(triples[3 * q + w])) return fail(FDTD_ERR_BADARG, "non-finite coefficient");
  }
  CK(cudaSetDevice(c->device));
  int* d_idx = nullptr;
  double* d_trip = nullptr;
  int rc = FDTD_OK;
  if (cudaMalloc((void**)&d_idx, count * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&d_trip, 3 * count * sizeof(double)) != cudaSuccess)
    rc = fail(FDTD_ERR_OOM, "override buffers");
  if (!rc && (xfer(c, d_idx, idx, count * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
              xfer(c, d_trip, triples, 3 * count * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess))
    rc = fail(FDTD_ERR_CUDA, "override upload");
  if (!rc) {
    k_coef_override<<<1, 1, 0, c->stream>>>((double*)c->coef[3 * comp], (double*)c->coef[3 * comp + 1],
                                            (double*)c->coef[3 * comp + 2], d_idx, d_trip, count);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess)
      rc = fail(FDTD_ERR_CUDA, "override: %s", cudaGetErrorString(cudaGetLastError()));
  }
  cudaFree(d_idx);
  cudaFree(d_trip);
  invalidate(c);
  return rc;
}

int fdtd_ctx_override_material(fdtd_ctx* c, int comp, const int* idx, const double* triples, int count) {
  if (!c || !idx || !triples) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (count > 0) {
    digest_vals(c, 10, {(double)comp, (double)count});
    digest(c, 10, idx, (size_t)count * sizeof(int));
    digest(c, 10, triples, (size_t)count * 3 * sizeof(double));
  }
  if (c->prec == FDTD_PREC_F64) return override_coef64(c, comp, idx, triples, count);
  if (c->prec != FDTD_PREC_F32_TABLE) return fail(FDTD_ERR_STATE, "not a material-table or FP64 problem");
  if (comp < 0 || comp > 5 || !c->ids_set[comp]) return fail(FDTD_ERR_STATE, "component %d has no material ids yet", comp);
  const long long n = c->ncomp[(comp + 3) % 6];
  std::vector<double> rows = c->rows64[comp];
  CK(cudaSetDevice(c->device));
  for (int q = 0; q < count; q++) {
    if (idx[q] < 0 || idx[q] >= n) return fail(FDTD_ERR_BADARG, "cell index %d out of range", idx[q]);
    int r = -1;
    for (size_t u = 0; u + 2 < rows.size(); u += 3)
      if (rows[u] == triples[3 * q] && rows[u + 1] == triples[3 * q + 1] && rows[u + 2] == triples[3 * q + 2]) r = (int)u / 3;
    if (r < 0) {
      r = (int)rows.size() / 3;
      rows.insert(rows.end(), triples + 3 * q, triples + 3 * q + 3);
    }
    if (r >= kTableRows) return fail(FDTD_ERR_BADARG, "component %d: coefficient rows exceed %d", comp, kTableRows);
    const uint8_t id = (uint8_t)r;
    CK(xfer(c, c->ids[comp] + idx[q], &id, 1, cudaMemcpyHostToDevice));
  }
  int rc = set_rows(c, comp, rows);
  invalidate(c);
  return rc;
}

int fdtd_ctx_read_material(fdtd_ctx* c, int comp, unsigned char* ids, long n, double* table, int* rows) {
  if (!c || !ids || !table || !rows) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (c->prec != FDTD_PREC_F32_TABLE || comp < 0 || comp > 5 || !c->ids_set[comp]) return fail(FDTD_ERR_STATE, "no material ids for component %d", comp);
  if (n != c->ncomp[(comp + 3) % 6]) return fail(FDTD_ERR_BADARG, "id buffer of %ld, need %lld", n, c->ncomp[(comp + 3) % 6]);
  CK(cudaSetDevice(c->device));
  CK(xfer(c, ids, c->ids[comp], n, cudaMemcpyDeviceToHost));
  *rows = (int)c->rows64[comp].size() / 3;
  std::copy(c->rows64[comp].begin(), c->rows64[comp].end(), table);
  return FDTD_OK;
}

int fdtd_ctx_run(fdtd_ctx* c, int count) {
  if (!c) return fail(FDTD_ERR_BADARG, "NULL handle");
  return run_steps(c, count);
}

int fdtd_ctx_set_prefetch(fdtd_ctx* c, int planes) {
  if (!c) return fail(FDTD_ERR_BADARG, "NULL handle");
  if (planes < 1 || planes > 5) return fail(FDTD_ERR_BADARG, "prefetch depth %d not in 1..5", planes);
  if (planes > 2 && c->prec != FDTD_PREC_F32_TABLE)
    return fail(FDTD_ERR_BADARG, "prefetch modes 3..5 (shared-memory stages) need a material-table problem");
  c->prefetch = planes;
  invalidate(c);
  return FDTD_OK;
}

int fdtd_ctx_set_tiling(fdtd_ctx* c, int x_planes_per_thread, int block_rows) {
  if (!c) return fail(FDTD_ERR_BADARG, "NULL handle");
  if (x_planes_per_thread < 1 || x_planes_per_thread > c->nx + 1)
    return fail(FDTD_ERR_BADARG, "x planes per thread %d not in 1..%d", x_planes_per_thread, c->nx + 1);
  if (block_rows != 1 && block_rows != 2 && block_rows != 4 && block_rows != 8 && block_rows != 16)
    return fail(FDTD_ERR_BADARG, "block rows %d not in {1,2,4,8,16}", block_rows);
  c->ichunk = x_planes_per_thread;
  c->block_rows = block_rows;
  invalidate(c);
  return FDTD_OK;
}

int fdtd_ctx_set_block_width(fdtd_ctx* c, int threads_along_k) {
  if (!c) return fail(FDTD_ERR_BADARG, "NULL handle");
  if (threads_along_k != 16 && threads_along_k != 32)
    return fail(FDTD_ERR_BADARG, "block width %d not 16 or 32", threads_along_k);
  c->block_w = threads_along_k;
  invalidate(c);
  return FDTD_OK;
}

int fdtd_ctx_get_block_width(const fdtd_ctx* c, int* threads_along_k) {
  if (!c || !threads_along_k) return fail(FDTD_ERR_BADARG, "NULL argument");
  *threads_along_k = c->block_w;
  return FDTD_OK;
}

int fdtd_ctx_get_tiling(const fdtd_ctx* c, int* x_planes_per_thread, int* block_rows) {
  if (!c || !x_planes_per_thread || !block_rows) return fail(FDTD_ERR_BADARG, "NULL argument");
  *x_planes_per_thread = c->ichunk;
  *block_rows = c->block_rows;
  return FDTD_OK;
}

int fdtd_ctx_run_timed(fdtd_ctx* c, int count, float* ms) {
  if (!c || !ms) return fail(FDTD_ERR_BADARG, "NULL argument");
  return run_steps(c, count, ms);
}

int fdtd_ctx_profile_kernels(fdtd_ctx* c, int count, double* avg_ms) {
  if (!c || !avg_ms || count < 1) return fail(FDTD_ERR_BADARG, "bad arguments");
  KernelTimer tm;
  CK(cudaSetDevice(c->device));
  for (int q = 0; q < 5; q++) CK(cudaEventCreate(&tm.ev[q]));
  int rc = run_steps(c, count, nullptr, &tm);
  for (int q = 0; q < 5; q++) cudaEventDestroy(tm.ev[q]);
  if (rc) return rc;
  for (int q = 0; q < 4; q++) avg_ms[q] = tm.ms[q] / count;
  return FDTD_OK;
}

int fdtd_ctx_step(const fdtd_ctx* c) { return c ? c->ts : -1; }

int fdtd_status(fdtd_ctx* c, int* code, int* step) {
  if (!c || !code || !step) return fail(FDTD_ERR_BADARG, "NULL argument");
  int st[2];
  CK(cudaSetDevice(c->device));
  CK(xfer(c, st, c->d_status, sizeof(st), cudaMemcpyDeviceToHost));
  *code = st[0];
  *step = st[0] ? st[1] : -1;
  return FDTD_OK;
}

int fdtd_ctx_read_trace(fdtd_ctx* c, int kind, int probe, double* out, int n) {
  if (!c || !out) return fail(FDTD_ERR_BADARG, "NULL argument");
  const int np = kind == 0 ? (int)c->vprobe.size() : (int)c->iprobe.size();
  if (kind < 0 || kind > 1 || probe < 0 || probe >= np) return fail(FDTD_ERR_BADARG, "no probe %d of kind %d", probe, kind);
  if (n < 0 || n > c->nsteps) return fail(FDTD_ERR_BADARG, "bad length %d", n);
  CK(cudaSetDevice(c->device));
  const double* src = (kind == 0 ? c->V : c->I) + (size_t)probe * c->nsteps;
  CK(xfer(c, out, src, n * sizeof(double), cudaMemcpyDeviceToHost));
  return FDTD_OK;
}

int fdtd_ctx_read_field(fdtd_ctx* c, int which, double* host, long n) {
  if (!c || !host) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (which < 0 || which > 5) return fail(FDTD_ERR_BADARG, "field id %d not in 0..5", which);
  if (n != c->ncomp[which]) return fail(FDTD_ERR_BADARG, "field %d: buffer of %ld, need %lld", which, n, c->ncomp[which]);
  CK(cudaSetDevice(c->device));
  return read_real(c, field_ptr(c, which), host, n);
}

int fdtd_ctx_read_psi(fdtd_ctx* c, int f, int slot, double* host, long n) {
  if (!c || !host) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (f < 0 || f > 5 || slot < 0 || slot > 3 || !c->face[f].present) return fail(FDTD_ERR_BADARG, "no Psi slot %d on face %d", slot, f);
  if (n != c->face[f].n[slot]) return fail(FDTD_ERR_BADARG, "Psi buffer of %ld, need %lld", n, c->face[f].n[slot]);
  CK(cudaSetDevice(c->device));
  return read_real(c, c->face[f].psi[slot], host, n);
}

int fdtd_ctx_read_farfield(fdtd_ctx* c, int array, double* re, double* im, long n) {
  if (!c || !re || !im) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (c->nFreq == 0) return fail(FDTD_ERR_STATE, "no far field set up");
  if (array < 0 || array > 23) return fail(FDTD_ERR_BADARG, "array %d not in 0..23", array);
  const long long m = c->nFreq * c->ffsz[(array % 12) / 4];
  if (n != m) return fail(FDTD_ERR_BADARG, "far-field buffer of %ld, need %lld", n, m);
  CK(cudaSetDevice(c->device));
  CK(xfer(c, re, c->acc + c->ffoff[array], m * sizeof(double), cudaMemcpyDeviceToHost));
  CK(xfer(c, im, c->acc + c->ffoff[array] + m, m * sizeof(double), cudaMemcpyDeviceToHost));
  if (c->acc_kahan) {
    // each 8-byte slot holds (sum, compensation) as two floats; the sum is sum - compensation
    for (double* a : {re, im})
      for (long long q = 0; q < m; q++) {
        float v[2];
        memcpy(v, &a[q], sizeof(v));
        a[q] = (double)v[0] - (double)v[1];
      }
  }
  return FDTD_OK;
}

// ---------------------------------------------------------------------------
// Checkpoint / restore of the evolving state: fields, Psi, port traces,
// far-field accumulators, watchdog and step.  The problem definition
// (coefficients, tables, sources, probes, boxes) is not part of it: a state
// loads into a handle set up with the same problem.
// ---------------------------------------------------------------------------
namespace {

struct StateHeader {
  char magic[8];  // "FDTDST2\0"
  int nx, ny, nz, prec, nsteps, ts, nv, ni, nfreq, kahan;
  long long psi[6][4];
  long long ff_values;
  unsigned long long setup;  // the handle's set-up digest
  long long bytes;  // whole state, header included
};

// The device ranges of a handle's state, in state order.
std::vector<std::pair<void*, size_t>> state_ranges(fdtd_ctx* c) {
  std::vector<std::pair<void*, size_t>> r;
  long long tot = 0;
  for (int q = 0; q < 6; q++) tot += c->ncomp[q];
  r.push_back({c->fields, (size_t)tot * c->esz});
  for (int f = 0; f < 6; f++)
    for (int s = 0; s < 4; s++)
      if (c->face[f].present && c->face[f].psi[s]) r.push_back({c->face[f].psi[s], (size_t)c->face[f].n[s] * c->esz});
  r.push_back({c->V, sizeof(double) * std::max((int)c->vprobe.size(), 1) * (size_t)c->nsteps});
  r.push_back({c->I, sizeof(double) * std::max((int)c->iprobe.size(), 1) * (size_t)c->nsteps});
  if (c->nFreq > 0) r.push_back({c->acc, sizeof(double) * (size_t)(c->ffoff[23] + 2LL * c->nFreq * c->ffsz[2])});
  r.push_back({c->d_status, 2 * sizeof(int)});
  return r;
}

StateHeader state_header(fdtd_ctx* c) {
  StateHeader h{};
  memcpy(h.magic, "FDTDST2", 8);
  h.nx = c->nx; h.ny = c->ny; h.nz = c->nz; h.prec = c->prec; h.nsteps = c->nsteps; h.ts = c->ts;
  h.nv = (int)c->vprobe.size(); h.ni = (int)c->iprobe.size(); h.nfreq = c->nFreq; h.kahan = c->acc_kahan;
  for (int f = 0; f < 6; f++)
    for (int s = 0; s < 4; s++) h.psi[f][s] = (c->face[f].present && c->face[f].psi[s]) ? c->face[f].n[s] : 0;
  h.ff_values = c->nFreq > 0 ? c->ffoff[23] + 2LL * c->nFreq * c->ffsz[2] : 0;
  h.setup = c->setup_digest;
  long long bytes = sizeof(StateHeader);
  for (auto& q : state_ranges(c)) bytes += (long long)q.second;
  h.bytes = bytes;
  return h;
}

}  // namespace

int fdtd_ctx_state_size(fdtd_ctx* c, long long* bytes) {
  if (!c || !bytes) return fail(FDTD_ERR_BADARG, "NULL argument");
  int rc = ensure_traces(c);
  if (rc) return rc;
  *bytes = state_header(c).bytes;
  return FDTD_OK;
}

int fdtd_ctx_save_state(fdtd_ctx* c, void* buf, long long bytes) {
  if (!c || !buf) return fail(FDTD_ERR_BADARG, "NULL argument");
  CK(cudaSetDevice(c->device));
  int rc = ensure_traces(c);
  if (rc) return rc;
  const StateHeader h = state_header(c);
  if (bytes != h.bytes) return fail(FDTD_ERR_BADARG, "state buffer of %lld bytes, need %lld", bytes, h.bytes);
  char* p = (char*)buf;
  memcpy(p, &h, sizeof(h));
  p += sizeof(h);
  for (auto& q : state_ranges(c)) {
    CK(cudaMemcpyAsync(p, q.first, q.second, cudaMemcpyDeviceToHost, c->stream));
    p += q.second;
  }
  CK(cudaStreamSynchronize(c->stream));
  return FDTD_OK;
}

int fdtd_ctx_load_state(fdtd_ctx* c, const void* buf, long long bytes) {
  if (!c || !buf) return fail(FDTD_ERR_BADARG, "NULL argument");
  CK(cudaSetDevice(c->device));
  int rc = ensure_traces(c);
  if (rc) return rc;
  StateHeader mine = state_header(c), theirs;
  if (bytes < (long long)sizeof(StateHeader)) return fail(FDTD_ERR_BADARG, "state buffer too small");
  memcpy(&theirs, buf, sizeof(theirs));
  if (memcmp(theirs.magic, "FDTDST2", 8) != 0) return fail(FDTD_ERR_BADARG, "not an engine state");
  mine.ts = theirs.ts;  // the step is what loading changes
  if (theirs.setup != mine.setup)
    return fail(FDTD_ERR_BADARG, "state was saved from a handle set up with other data (grid, dt, coefficients, "
                                 "faces, sources, probes or far field)");
  if (memcmp(&mine, &theirs, sizeof(StateHeader)) != 0 || bytes != theirs.bytes)
    return fail(FDTD_ERR_BADARG, "state was saved from a problem of another shape, precision or probe set");
  if (theirs.ts < 0 || theirs.ts > c->nsteps) return fail(FDTD_ERR_BADARG, "state step %d out of range", theirs.ts);
  const char* p = (const char*)buf + sizeof(StateHeader);
  for (auto& q : state_ranges(c)) {
    CK(cudaMemcpyAsync(q.first, p, q.second, cudaMemcpyHostToDevice, c->stream));
    p += q.second;
  }
  const int dts = theirs.ts - 1;  // the device counter holds the index of the last step run
  CK(cudaMemcpyAsync(c->d_ts, &dts, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  if (c->d_dft_done)  // a saved state has no open DFT block
    CK(cudaMemcpyAsync(c->d_dft_done, &theirs.ts, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->ts = theirs.ts;
  return FDTD_OK;
}

int fdtd_ctx_set_dft_block(fdtd_ctx* c, int steps) {
  if (!c) return fail(FDTD_ERR_BADARG, "NULL handle");
  if (steps < 0 || steps == 1 || steps > 1024) return fail(FDTD_ERR_BADARG, "DFT block of %d steps not in {0, 2..1024}", steps);
  if (steps && c->prec == FDTD_PREC_F64) return fail(FDTD_ERR_BADARG, "FP64 problems keep the per-step DFT");
  if (steps && c->nFreq == 0) return fail(FDTD_ERR_STATE, "no far field set up");
  CK(cudaSetDevice(c->device));
  if (steps) {
    dfree(c, c->dft_samples);
    c->dft_samples = nullptr;
    const long long npts = c->ffsz[0] + c->ffsz[1] + c->ffsz[2];
    int rc = dalloc(c, (void**)&c->dft_samples, sizeof(float) * (size_t)steps * npts * 8);
    if (!rc && !c->d_dft_done) rc = dalloc(c, (void**)&c->d_dft_done, sizeof(int));
    if (rc) return rc;
    // every earlier step is already in the accumulators
    CK(xfer(c, c->d_dft_done, &c->ts, sizeof(int), cudaMemcpyHostToDevice));
  }
  c->dft_block = steps;
  invalidate(c);
  return FDTD_OK;
}

int fdtd_ctx_set_dft_accumulator(fdtd_ctx* c, int kahan_fp32) {
  if (!c) return fail(FDTD_ERR_BADARG, "NULL handle");
  if (kahan_fp32 != 0 && kahan_fp32 != 1) return fail(FDTD_ERR_BADARG, "accumulator mode %d not in {0,1}", kahan_fp32);
  if (kahan_fp32 && c->prec == FDTD_PREC_F64) return fail(FDTD_ERR_BADARG, "FP64 problems keep FP64 accumulators");
  if (c->ts != 0) return fail(FDTD_ERR_STATE, "the accumulator mode is set before the first step");
  c->acc_kahan = kahan_fp32;
  invalidate(c);
  return FDTD_OK;
}

int fdtd_ctx_set_x_wall(fdtd_ctx* c, int wall) {
  if (!c) return fail(FDTD_ERR_BADARG, "NULL handle");
  if (wall != 0 && wall != 1) return fail(FDTD_ERR_BADARG, "x wall mode %d not in {0,1}", wall);
  c->x_wall = wall;
  invalidate(c);
  return FDTD_OK;
}

int fdtd_ctx_get_x_wall(const fdtd_ctx* c, int* wall) {
  if (!c || !wall) return fail(FDTD_ERR_BADARG, "NULL argument");
  *wall = c->x_wall;
  return FDTD_OK;
}

// Direct time-to-frequency transform (dft.js:17-38); one block per frequency.
__global__ void __launch_bounds__(256) k_dft(const double* x, int N, double dt, const double* f, double shift,
                                             double* re, double* im) {
  __shared__ double sr[256], si[256];
  const int m = blockIdx.x;
  const double w = 2 * M_PI * f[m];
  double r = 0.0, q = 0.0;
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    const double ph = w * ((n + 1) * dt + shift);
    double s, c;
    sincos(ph, &s, &c);
    r += x[n] * c;
    q -= x[n] * s;
  }
  sr[threadIdx.x] = r;
  si[threadIdx.x] = q;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sr[threadIdx.x] += sr[threadIdx.x + o];
      si[threadIdx.x] += si[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    re[m] = sr[0] * dt;
    im[m] = si[0] * dt;
  }
}

int fdtd_dft(const double* x, int N, double dt, const double* freqs, int M, double shift, double* re, double* im) {
  if (!x || !freqs || !re || !im || N <= 0 || M <= 0) return fail(FDTD_ERR_BADARG, "bad DFT arguments");
  double *dx_ = nullptr, *df = nullptr, *dr = nullptr;
  int rc = FDTD_OK;
  if (cudaMalloc(&dx_, N * sizeof(double)) != cudaSuccess || cudaMalloc(&df, M * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&dr, 2 * M * sizeof(double)) != cudaSuccess) {
    rc = fail(FDTD_ERR_OOM, "DFT buffers");
  } else if (cudaMemcpy(dx_, x, N * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
             cudaMemcpy(df, freqs, M * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    rc = fail(FDTD_ERR_CUDA, "DFT upload");
  } else {
    k_dft<<<M, 256>>>(dx_, N, dt, df, shift, dr, dr + M);
    if (cudaMemcpy(re, dr, M * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(im, dr + M, M * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = fail(FDTD_ERR_CUDA, "DFT: %s", cudaGetErrorString(cudaGetLastError()));
  }
  cudaFree(dx_);
  cudaFree(df);
  cudaFree(dr);
  return rc;
}

int fdtd_ctx_farfield_post(fdtd_ctx* c, const double* theta, const double* phi, int nang, double* radp,
                           double* d_theta, double* d_phi) {
  if (!c || !radp || (nang > 0 && (!theta || !phi || !d_theta || !d_phi)) || nang < 0)
    return fail(FDTD_ERR_BADARG, "bad far-field post arguments");
  if (c->nFreq == 0) return fail(FDTD_ERR_STATE, "no far field set up");
  CK(cudaSetDevice(c->device));
  FFPost P{};
  P.acc = c->acc;
  double* conv = nullptr;
  if (c->acc_kahan) {
    const long long n = c->ffoff[23] + 2LL * c->nFreq * c->ffsz[2];
    if (cudaMalloc(&conv, n * sizeof(double)) != cudaSuccess) return fail(FDTD_ERR_OOM, "far-field post buffer");
    k_kahan_to_f64<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->acc, conv, n);
    P.acc = conv;
  }
  for (int a = 0; a < 24; a++) P.off[a] = c->ffoff[a];
  for (int a = 0; a < 3; a++) P.sz[a] = c->ffsz[a];
  P.nFreq = c->nFreq;
  P.ni = c->ui - c->li;
  P.nj = c->uj - c->lj;
  P.nk = c->uk - c->lk;
  const double d[3] = {c->dx, c->dy, c->dz};
  const int lo[3] = {c->li, c->lj, c->lk}, hi[3] = {c->ui, c->uj, c->uk};
  for (int a = 0; a < 3; a++) {
    const double centre = 0.5 * (hi[a] + lo[a]);
    P.d[a] = d[a];
    P.pos0[a] = ((lo[a] - 1) - centre + 0.5) * d[a];
    P.face[a][0] = (hi[a] - centre) * d[a];
    P.face[a][1] = (lo[a] - centre) * d[a];
  }
  const int F = c->nFreq;
  double *dfreq = nullptr, *dradp = nullptr, *dang = nullptr, *dout = nullptr;
  int rc = FDTD_OK;
  const size_t na = (size_t)std::max(nang, 1);
  if (cudaMalloc(&dfreq, F * sizeof(double)) != cudaSuccess || cudaMalloc(&dradp, F * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&dang, 2 * na * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&dout, 2 * F * na * sizeof(double)) != cudaSuccess) {
    rc = fail(FDTD_ERR_OOM, "far-field post buffers");
  }
  cudaError_t e = cudaSuccess;
  if (!rc) {
    e = cudaMemcpyAsync(dfreq, c->ffreq.data(), F * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nang > 0)
      e = cudaMemcpyAsync(dang, theta, nang * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nang > 0)
      e = cudaMemcpyAsync(dang + na, phi, nang * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
      k_ff_power<<<F, 256, 0, c->stream>>>(P, dradp);
      if (nang > 0) {
        const dim3 grd((nang + 256 * kFFAng - 1) / (256 * kFFAng), F);
        k_ff_pattern<<<grd, 256, 0, c->stream>>>(P, dfreq, dang, dang + na, nang, dradp, dout, dout + F * na);
      }
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(radp, dradp, F * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && nang > 0)
      for (int f = 0; f < F && e == cudaSuccess; f++) {
        e = cudaMemcpyAsync(d_theta + (size_t)f * nang, dout + f * na, nang * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(d_phi + (size_t)f * nang, dout + F * na + f * na, nang * sizeof(double),
                              cudaMemcpyDeviceToHost, c->stream);
      }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) rc = fail(FDTD_ERR_CUDA, "far-field post: %s", cudaGetErrorString(e));
  }
  cudaFree(dfreq);
  cudaFree(dradp);
  cudaFree(dang);
  cudaFree(dout);
  cudaFree(conv);
  return rc;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of fdtd_dft.  Its device staging area is this
// file-scope array instead of cudaMalloc'd buffers, so a call allocates and
// frees nothing.  Every GPU that loads the library holds the array until the
// process exits.  Layout: samples | frequencies | re | im.
// ---------------------------------------------------------------------------
constexpr int kDftNoAllocMaxSamples = 32768;
constexpr int kDftNoAllocMaxFreqs = 4096;
static __device__ __align__(256) double g_dft_scratch[kDftNoAllocMaxSamples + 3 * kDftNoAllocMaxFreqs];

// The array's device address, looked up once per device with that device
// current.  In host code `g_dft_scratch` only names a host-side stand-in, so
// the kernel must be given this address, never the symbol itself.
static int dft_scratch_address(double** out) {
  constexpr int kMaxDevices = 64;
  static double* addr[kMaxDevices] = {};
  static std::mutex lock;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(FDTD_ERR_CUDA, "device ordinal %d not supported", dev);
  std::lock_guard<std::mutex> g(lock);
  if (!addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_dft_scratch);
    if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, "cudaGetSymbolAddress(dft scratch): %s", cudaGetErrorString(e));
    addr[dev] = (double*)p;
  }
  *out = addr[dev];
  return FDTD_OK;
}

int fdtd_dft_noalloc(const double* x, int N, double dt, const double* freqs, int M, double shift, double* re,
                     double* im) {
  if (!x || !freqs || !re || !im) return fail(FDTD_ERR_BADARG, "NULL argument");
  if (N <= 0 || N > kDftNoAllocMaxSamples)
    return fail(FDTD_ERR_BADARG, "fdtd_dft_noalloc: %d samples, must be 1..%d", N, kDftNoAllocMaxSamples);
  if (M <= 0 || M > kDftNoAllocMaxFreqs)
    return fail(FDTD_ERR_BADARG, "fdtd_dft_noalloc: %d frequencies, must be 1..%d", M, kDftNoAllocMaxFreqs);
  double* s = nullptr;
  int rc = dft_scratch_address(&s);
  if (rc) return rc;
  double* d_x = s;
  double* d_f = s + kDftNoAllocMaxSamples;
  double* d_re = d_f + kDftNoAllocMaxFreqs;
  double* d_im = d_re + kDftNoAllocMaxFreqs;
  // Every value the kernel reads is written by this call and every output is
  // fully overwritten, so nothing left by an earlier call needs clearing.
  CK(cudaMemcpy(d_x, x, N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_f, freqs, M * sizeof(double), cudaMemcpyHostToDevice));
  k_dft<<<M, 256>>>(d_x, N, dt, d_f, shift, d_re, d_im);
  CK(cudaGetLastError());
  CK(cudaMemcpy(re, d_re, M * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(im, d_im, M * sizeof(double), cudaMemcpyDeviceToHost));
  return FDTD_OK;
}

}  // extern "C"

// ===========================================================================
// Batches: member handles advanced together, one launch per kernel kind per
// step for all of them (fdtd_batch.cuh).
// ===========================================================================
struct fdtd_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int prec = FDTD_PREC_F32_TABLE;
  std::vector<fdtd_ctx*> m;
  int ichunk = 8, block_rows = 4, prefetch = 1, group = 0;
  int block_w = 32;
  void* d_inst = nullptr;
  size_t inst_size = 0;  // bytes of one Instance
  BatchTile* d_tiles = nullptr;
  BatchBlock* d_mid = nullptr;
  BatchBlock* d_epi = nullptr;
  BatchCtl* d_ctl = nullptr;
  std::vector<BatchTile> tiles;
  std::vector<BatchBlock> mid, epi, flush;
  BatchBlock* d_flush = nullptr;
  int grid_h = 0, grid_e = 0;  // persistent grid sizes
  RunGraphs graphs;
  // member-kernel mode (streams > 0): each member's own step kernels, members
  // spread over `streams` worker streams joined to `stream`
  int streams = 0;
  std::vector<cudaStream_t> ws;
  std::vector<cudaEvent_t> wev;
  cudaEvent_t fork_ev = nullptr;
  // grouped mode (members_per_launch > 0, streams == 0): the members'
  // parameter blocks travel as kernel parameters, `members_per_launch` per
  // launch; the launches of one half-step run side by side on worker streams
  int members_per_launch = 0;
  std::vector<unsigned char> groups;  // host copies of the BatchGroup parameter structs
  int ngroups = 0;
  size_t group_size = 0;
};

namespace {

void batch_drop_graph(fdtd_batch* b) { b->graphs.clear(); }

template <class V>
int upload_vec(fdtd_batch* b, V** dst, const std::vector<V>& v) {
  if (*dst) cudaFree(*dst);
  *dst = nullptr;
  const size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(V);
  CK(cudaMalloc((void**)dst, bytes));
  if (!v.empty()) CK(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return FDTD_OK;
}

// Batched H/E kernel for a prefetch depth (as step_kernel) and grid kind.
template <typename T, class C, bool EXACT>
void (*batch_kernel(bool electric, int pf, bool persist))(const Instance<T, C>*, const BatchTile*, int, BatchCtl*,
                                                           int) {
#define FDTD_BK(PF)                                                                                           \
  (electric ? (persist ? k_batch_half<T, C, EXACT, PF, true, true> : k_batch_half<T, C, EXACT, PF, true, false>) \
            : (persist ? k_batch_half<T, C, EXACT, PF, false, true> : k_batch_half<T, C, EXACT, PF, false, false>))
  if constexpr (C::kTable) {
    if (pf == 3) return FDTD_BK(3);
    if (pf == 4) return FDTD_BK(4);
  }
  if (pf == 2) return FDTD_BK(2);
  return FDTD_BK(1);
#undef FDTD_BK
}

// Grouped H/E kernel for a prefetch depth (as step_kernel).
template <typename T, class C, bool EXACT>
void (*batch_group_kernel(bool electric, int pf))(const BatchGroup<T, C>) {
#define FDTD_GK(PF) (electric ? k_batch_group<T, C, EXACT, PF, true> : k_batch_group<T, C, EXACT, PF, false>)
  if constexpr (C::kTable) {
    if (pf == 3) return FDTD_GK(3);
    if (pf == 4) return FDTD_GK(4);
  }
  if (pf == 2) return FDTD_GK(2);
  return FDTD_GK(1);
#undef FDTD_GK
}

int batch_worker_streams(fdtd_batch* b, int count);

// One half-step of every group: the groups' launches fork from the batch's
// stream onto worker streams and join back into it (also under capture).
template <typename T, class C, bool EXACT>
int batch_group_half(fdtd_batch* b, bool electric, size_t smem) {
  using G = BatchGroup<T, C>;
  auto k = batch_group_kernel<T, C, EXACT>(electric, b->prefetch);
  const dim3 blk(b->block_w, b->block_rows);
  CK(cudaEventRecord(b->fork_ev, b->stream));
  for (int g = 0; g < b->ngroups; g++) {
    const G& grp = *reinterpret_cast<const G*>(b->groups.data() + (size_t)g * sizeof(G));
    cudaStream_t st = b->ngroups == 1 ? b->stream : b->ws[g];
    if (st != b->stream) CK(cudaStreamWaitEvent(st, b->fork_ev, 0));
    k<<<(unsigned)grp.first[grp.n], blk, smem, st>>>(grp);
    if (st != b->stream) {
      CK(cudaEventRecord(b->wev[g], st));
      CK(cudaStreamWaitEvent(b->stream, b->wev[g], 0));
    }
  }
  CK(cudaGetLastError());
  return FDTD_OK;
}

// The parameter blocks of every member (member state may have moved since the
// last run: traces, tables) and, when the work lists changed, the lists.
template <typename T, class C, bool EXACT>
int batch_prepare(fdtd_batch* b, C (*coef_of)(fdtd_ctx*)) {
  using In = Instance<T, C>;
  const int n = (int)b->m.size();
  std::vector<unsigned char> host((size_t)n * sizeof(In), 0);
  std::vector<BatchTile> tiles;
  std::vector<BatchBlock> mid, epi, flush;
  for (int q = 0; q < n; q++) {
    fdtd_ctx* c = b->m[q];
    In in;
    memset(&in, 0, sizeof(In));
    in.sp = step_params<T, C>(c, coef_of(c));
    in.sp.ichunk = b->ichunk;
    in.sp.ts = &b->d_ctl->ts;
    in.pr = dev_probes(c);
    in.ff = dev_ff(c);
    memcpy(host.data() + (size_t)q * sizeof(In), &in, sizeof(In));
    const int gx = (c->nz + b->block_w) / b->block_w, gy = (c->ny + b->block_rows) / b->block_rows,
              gz = (c->nx + 1 + b->ichunk - 1) / b->ichunk;
    if (gx > 65535 || gy > 65535 || gz > 65535)
      return fail(FDTD_ERR_BADARG, "batch member %d: %dx%dx%d tiles exceed the tile index range", q, gx, gy, gz);
    for (int z = 0; z < gz; z++)
      for (int y = 0; y < gy; y++)
        for (int x = 0; x < gx; x++)
          tiles.push_back(BatchTile{(unsigned short)q, (unsigned short)x, (unsigned short)y, (unsigned short)z});
    const long long nmid = (long long)c->ny * (c->nz + 1) + in.pr.n_i;
    for (long long s = 0; s < (nmid + 255) / 256; s++) mid.push_back(BatchBlock{q, (int)s});
    const long long nff = (c->nFreq > 0) ? c->ffsz[0] + c->ffsz[1] + c->ffsz[2] : 0;
    for (long long s = 0; s < (nff + in.pr.n_v + 255) / 256; s++) epi.push_back(BatchBlock{q, (int)s});
    if (c->dft_block > 0)
      for (long long s = 0; s < (nff * c->nFreq + 255) / 256; s++) flush.push_back(BatchBlock{q, (int)s});
  }
  if (tiles.size() > (size_t)INT32_MAX) return fail(FDTD_ERR_BADARG, "batch has too many tiles");
  if (b->members_per_launch > 0) {
    // grouped mode: consecutive members, members_per_launch per launch
    using G = BatchGroup<T, C>;
    const int per = b->members_per_launch;
    const int ng = (n + per - 1) / per;
    std::vector<unsigned char> gbytes((size_t)ng * sizeof(G), 0);
    for (int g = 0; g < ng; g++) {
      G grp;
      memset(&grp, 0, sizeof(G));
      grp.ts = g == 0 ? &b->d_ctl->ts : nullptr;
      long long blocks = 0;
      for (int q = g * per; q < std::min(n, (g + 1) * per); q++) {
        fdtd_ctx* c = b->m[q];
        const int k = q - g * per;
        const int gx = (c->nz + b->block_w) / b->block_w, gy = (c->ny + b->block_rows) / b->block_rows,
                  gz = (c->nx + 1 + b->ichunk - 1) / b->ichunk;
        grp.first[k] = (int)blocks;
        grp.gx[k] = gx;
        grp.gy[k] = gy;
        memcpy(&grp.sp[k], host.data() + (size_t)q * sizeof(In) + offsetof(In, sp), sizeof(grp.sp[k]));
        blocks += (long long)gx * gy * gz;
        grp.n = k + 1;
      }
      if (blocks > INT32_MAX) return fail(FDTD_ERR_BADARG, "batch group %d has too many blocks", g);
      grp.first[grp.n] = (int)blocks;
      memcpy(gbytes.data() + (size_t)g * sizeof(G), &grp, sizeof(G));
    }
    if (gbytes != b->groups) batch_drop_graph(b);
    b->groups.swap(gbytes);
    b->ngroups = ng;
    b->group_size = sizeof(G);
  } else {
    b->groups.clear();
    b->ngroups = 0;
  }
  if (!b->d_inst || b->inst_size != sizeof(In)) {
    if (b->d_inst) cudaFree(b->d_inst);
    b->d_inst = nullptr;
    CK(cudaMalloc(&b->d_inst, host.size()));
    b->inst_size = sizeof(In);
  }
  CK(cudaMemcpyAsync(b->d_inst, host.data(), host.size(), cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  auto same = [](const std::vector<BatchBlock>& u, const std::vector<BatchBlock>& v) {
    return u.size() == v.size() && (u.empty() || !memcmp(u.data(), v.data(), u.size() * sizeof(BatchBlock)));
  };
  const bool same_tiles = tiles.size() == b->tiles.size() &&
                          (tiles.empty() || !memcmp(tiles.data(), b->tiles.data(), tiles.size() * sizeof(BatchTile)));
  if (!same_tiles || !same(mid, b->mid) || !same(epi, b->epi) || !same(flush, b->flush) || !b->d_tiles) {
    batch_drop_graph(b);
    b->tiles.swap(tiles);
    b->mid.swap(mid);
    b->epi.swap(epi);
    b->flush.swap(flush);
    int rc = upload_vec(b, &b->d_tiles, b->tiles);
    if (!rc) rc = upload_vec(b, &b->d_mid, b->mid);
    if (!rc) rc = upload_vec(b, &b->d_epi, b->epi);
    if (!rc) rc = upload_vec(b, &b->d_flush, b->flush);
    if (rc) return rc;
  }
  // persistent grids: as many blocks as fit on the device at once
  int sms = 0, per_h = 0, per_e = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  int rc0 = check_block(b->block_w, b->block_rows);
  if (rc0) return rc0;
  const int threads = b->block_w * b->block_rows;
  size_t smem = 0;
  auto kh = batch_kernel<T, C, EXACT>(false, b->prefetch, true);
  auto ke = batch_kernel<T, C, EXACT>(true, b->prefetch, true);
  int rc = stage_smem(kh, b->prefetch, threads, &smem);
  if (!rc) rc = stage_smem(ke, b->prefetch, threads, &smem);
  if (rc) return rc;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_h, kh, threads, smem));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_e, ke, threads, smem));
  b->grid_h = std::max(1, per_h) * sms;
  b->grid_e = std::max(1, per_e) * sms;
  return FDTD_OK;
}

template <typename T, class C, bool EXACT>
int batch_enqueue(fdtd_batch* b, int count, KernelTimer* tm = nullptr) {
  const Instance<T, C>* in = (const Instance<T, C>*)b->d_inst;
  const int nt = (int)b->tiles.size();
  const dim3 blk(b->block_w, b->block_rows);
  const unsigned gh = b->group ? (unsigned)std::min(b->grid_h, (nt + b->group - 1) / b->group) : (unsigned)nt;
  const unsigned ge = b->group ? (unsigned)std::min(b->grid_e, (nt + b->group - 1) / b->group) : (unsigned)nt;
  auto kh = batch_kernel<T, C, EXACT>(false, b->prefetch, b->group != 0);
  auto ke = batch_kernel<T, C, EXACT>(true, b->prefetch, b->group != 0);
  size_t smem = 0;
  int rc = stage_smem(kh, b->prefetch, b->block_w * b->block_rows, &smem);
  if (!rc) rc = stage_smem(ke, b->prefetch, b->block_w * b->block_rows, &smem);
  if (rc) return rc;
  const bool grouped = b->ngroups > 0;
  size_t gsmem = 0;
  if (grouped) {
    rc = batch_worker_streams(b, b->ngroups);
    if (!rc) rc = stage_smem(batch_group_kernel<T, C, EXACT>(false, b->prefetch), b->prefetch,
                             b->block_w * b->block_rows, &gsmem);
    if (!rc) rc = stage_smem(batch_group_kernel<T, C, EXACT>(true, b->prefetch), b->prefetch,
                             b->block_w * b->block_rows, &gsmem);
    if (rc) return rc;
  }
  for (int s = 0; s < count; s++) {
    if (tm) CK(cudaEventRecord(tm->ev[0], b->stream));
    if (grouped) {
      rc = batch_group_half<T, C, EXACT>(b, false, gsmem);
      if (rc) return rc;
    } else {
      kh<<<gh, blk, smem, b->stream>>>(in, b->d_tiles, nt, b->d_ctl, b->group);
    }
    if (tm) CK(cudaEventRecord(tm->ev[1], b->stream));
    k_batch_mid<T, C, EXACT><<<(unsigned)b->mid.size(), 256, 0, b->stream>>>(in, b->d_mid, b->d_ctl,
                                                                             (int)b->m.size());
    if (tm) CK(cudaEventRecord(tm->ev[2], b->stream));
    if (grouped) {
      rc = batch_group_half<T, C, EXACT>(b, true, gsmem);
      if (rc) return rc;
    } else {
      ke<<<ge, blk, smem, b->stream>>>(in, b->d_tiles, nt, b->d_ctl, b->group);
    }
    if (tm) CK(cudaEventRecord(tm->ev[3], b->stream));
    if (!b->epi.empty()) k_batch_epilogue<T, C><<<(unsigned)b->epi.size(), 256, 0, b->stream>>>(in, b->d_epi);
    if (!b->flush.empty())
      k_batch_flush<T, C><<<(unsigned)b->flush.size(), 256, 0, b->stream>>>(in, b->d_flush, -1);
    if (tm) {
      CK(cudaEventRecord(tm->ev[4], b->stream));
      CK(cudaEventSynchronize(tm->ev[4]));
      for (int q = 0; q < 4; q++) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, tm->ev[q], tm->ev[q + 1]));
        tm->ms[q] += ms;
      }
    }
  }
  CK(cudaGetLastError());
  return FDTD_OK;
}

ArrayCoef<double> coef_f64(fdtd_ctx* c) { return array_coef<double>(c); }
ArrayCoef<float> coef_f32(fdtd_ctx* c) { return array_coef<float>(c); }
TableCoef coef_table(fdtd_ctx* c) { return c->tcoef; }

int batch_prepare_any(fdtd_batch* b) {
  if (b->prec == FDTD_PREC_F64) return batch_prepare<double, ArrayCoef<double>, true>(b, coef_f64);
  if (b->prec == FDTD_PREC_F32) return batch_prepare<float, ArrayCoef<float>, true>(b, coef_f32);
  return batch_prepare<float, TableCoef, false>(b, coef_table);
}

// Closes the members' open DFT blocks at the end of a run reaching `upto`.
template <typename T, class C>
int batch_close_blocks(fdtd_batch* b, int upto) {
  if (b->flush.empty()) return FDTD_OK;
  k_batch_flush<T, C><<<(unsigned)b->flush.size(), 256, 0, b->stream>>>((const Instance<T, C>*)b->d_inst, b->d_flush,
                                                                        upto);
  CK(cudaGetLastError());
  for (fdtd_ctx* c : b->m)
    if (c->dft_block > 0) CK(cudaMemcpyAsync(c->d_dft_done, &upto, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return FDTD_OK;
}

int batch_close_any(fdtd_batch* b, int upto) {
  if (b->prec == FDTD_PREC_F64) return batch_close_blocks<double, ArrayCoef<double>>(b, upto);
  if (b->prec == FDTD_PREC_F32) return batch_close_blocks<float, ArrayCoef<float>>(b, upto);
  return batch_close_blocks<float, TableCoef>(b, upto);
}

int batch_enqueue_any(fdtd_batch* b, int count, KernelTimer* tm = nullptr) {
  if (b->prec == FDTD_PREC_F64) return batch_enqueue<double, ArrayCoef<double>, true>(b, count, tm);
  if (b->prec == FDTD_PREC_F32) return batch_enqueue<float, ArrayCoef<float>, true>(b, count, tm);
  return batch_enqueue<float, TableCoef, false>(b, count, tm);
}

// Member-kernel mode.  Sets a member's launch shape to the batch's for the
// duration of a scope (its own shape comes back afterwards).
struct MemberShape {
  fdtd_ctx* c;
  int ichunk, rows, pf, w;
  MemberShape(fdtd_ctx* m, const fdtd_batch* b)
      : c(m), ichunk(m->ichunk), rows(m->block_rows), pf(m->prefetch), w(m->block_w) {
    m->ichunk = b->ichunk;
    m->block_rows = b->block_rows;
    m->prefetch = b->prefetch;
    m->block_w = b->block_w;
  }
  ~MemberShape() {
    c->ichunk = ichunk;
    c->block_rows = rows;
    c->prefetch = pf;
    c->block_w = w;
  }
};

int batch_worker_streams(fdtd_batch* b, int count) {
  while ((int)b->ws.size() < count) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    b->ws.push_back(st);
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->wev.push_back(ev);
  }
  if (!b->fork_ev) CK(cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming));
  return FDTD_OK;
}

// `count` steps of every member, member-major: worker stream s steps members
// s, s + S, s + 2S, ... one after another, all `count` steps of one member
// before the next, so a member's arrays are still in L2 at its next step.
// The worker streams fork from and join back into the batch's stream (also
// under stream capture), and are joined even when an enqueue fails.
int batch_member_enqueue(fdtd_batch* b, int count) {
  const int S = b->streams;
  CK(cudaEventRecord(b->fork_ev, b->stream));
  for (int q = 0; q < S; q++) CK(cudaStreamWaitEvent(b->ws[q], b->fork_ev, 0));
  int rc = FDTD_OK;
  for (size_t q = 0; q < b->m.size() && !rc; q++) {
    MemberShape shape(b->m[q], b);
    rc = enqueue(b->m[q], count, nullptr, b->ws[q % S]);
  }
  for (int q = 0; q < S; q++) {
    CK(cudaEventRecord(b->wev[q], b->ws[q]));
    CK(cudaStreamWaitEvent(b->stream, b->wev[q], 0));
  }
  return rc;
}

int batch_run_members(fdtd_batch* b, int count, float* elapsed_ms, KernelTimer* tm) {
  const int ts = b->m[0]->ts;
  int rc = batch_worker_streams(b, b->streams);
  if (rc) return rc;
  // the whole run as cached graphs, captured before the first launch
  std::vector<cudaGraphExec_t> plan;
  if (!tm) {
    int per_step = 0;
    for (fdtd_ctx* c : b->m) per_step += c->dft_block > 0 ? 5 : 4;
    rc = run_plan(b->graphs, b->stream, count, per_step, [b](int n) { return batch_member_enqueue(b, n); }, &plan);
    if (rc) return rc;
  }
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (elapsed_ms) {
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    CK(cudaEventRecord(ev0, b->stream));
  }
  if (tm) {
    // one member at a time on the batch's stream: per-kernel times summed over members
    for (size_t q = 0; q < b->m.size() && !rc; q++) {
      MemberShape shape(b->m[q], b);
      rc = enqueue(b->m[q], count, tm, b->stream);
    }
    if (rc) return rc;
  }
  for (cudaGraphExec_t ge : plan) CK(cudaGraphLaunch(ge, b->stream));
  if (elapsed_ms) {
    CK(cudaEventRecord(ev1, b->stream));
    CK(cudaEventSynchronize(ev1));
    CK(cudaEventElapsedTime(elapsed_ms, ev0, ev1));
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
  }
  for (fdtd_ctx* c : b->m) {
    rc = count > 0 ? close_dft_block(c, ts + count, b->stream) : FDTD_OK;
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(b->stream));
  for (fdtd_ctx* c : b->m) c->ts += count;
  for (size_t q = 0; q < b->m.size(); q++) {
    int st[2];
    CK(cudaMemcpyAsync(st, b->m[q]->d_status, sizeof(st), cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    if (st[0] != 0) return fail(FDTD_ERR_NONFINITE, "batch member %zu: non-finite port sample at step %d", q, st[1]);
  }
  return FDTD_OK;
}

int batch_run(fdtd_batch* b, int count, float* elapsed_ms = nullptr, KernelTimer* tm = nullptr) {
  if (count < 0) return fail(FDTD_ERR_BADARG, "negative step count %d", count);
  const int ts = b->m[0]->ts;
  for (size_t q = 0; q < b->m.size(); q++) {
    fdtd_ctx* c = b->m[q];
    if (c->ts != ts) return fail(FDTD_ERR_STATE, "batch member %zu is at step %d, member 0 at step %d", q, c->ts, ts);
    if (ts + count > c->nsteps)
      return fail(FDTD_ERR_BADARG, "batch member %zu: running %d steps from step %d exceeds numberOfTimeSteps=%d", q,
                  count, ts, c->nsteps);
    int rc = check_ready(c);
    if (!rc) rc = ensure_traces(c);
    if (!rc && c->prec == FDTD_PREC_F32_TABLE && c->table_dirty) rc = prepare_table(c, &c->tcoef);
    if (rc) {
      std::string msg = g_err;
      return fail(rc, "batch member %zu: %s", q, msg.c_str());
    }
  }
  CK(cudaSetDevice(b->device));
  if (b->streams > 0) return batch_run_members(b, count, elapsed_ms, tm);
  int rc = batch_prepare_any(b);
  if (rc) return rc;
  const int ctl_ts = ts - 1;
  CK(cudaMemcpyAsync(&b->d_ctl->ts, &ctl_ts, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  // the whole run as cached graphs, captured before the first launch
  std::vector<cudaGraphExec_t> plan;
  if (!tm) {
    const int per_step = (b->flush.empty() ? 2 : 3) + (b->ngroups > 0 ? 2 * b->ngroups : 2);
    rc = run_plan(b->graphs, b->stream, count, per_step, [b](int n) { return batch_enqueue_any(b, n); }, &plan);
    if (rc) return rc;
  }
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (elapsed_ms) {
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    CK(cudaEventRecord(ev0, b->stream));
  }
  if (tm) {
    rc = batch_enqueue_any(b, count, tm);
    if (rc) return rc;
  }
  for (cudaGraphExec_t ge : plan) CK(cudaGraphLaunch(ge, b->stream));
  if (elapsed_ms) {
    CK(cudaEventRecord(ev1, b->stream));
    CK(cudaEventSynchronize(ev1));
    CK(cudaEventElapsedTime(elapsed_ms, ev0, ev1));
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
  }
  if (count > 0) {
    rc = batch_close_any(b, ts + count);
    if (rc) return rc;
  }
  // hand the shared step counter back to every member
  for (fdtd_ctx* c : b->m) CK(cudaMemcpyAsync(c->d_ts, &b->d_ctl->ts, sizeof(int), cudaMemcpyDeviceToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  for (fdtd_ctx* c : b->m) c->ts += count;
  for (size_t q = 0; q < b->m.size(); q++) {
    int st[2];
    CK(cudaMemcpyAsync(st, b->m[q]->d_status, sizeof(st), cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    if (st[0] != 0) return fail(FDTD_ERR_NONFINITE, "batch member %zu: non-finite port sample at step %d", q, st[1]);
  }
  return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_batch_create(fdtd_ctx* const* members, int count, fdtd_batch** out) {
  if (!members || !out || count < 1) return fail(FDTD_ERR_BADARG, "bad batch arguments");
  *out = nullptr;
  if (count > 65535) return fail(FDTD_ERR_BADARG, "a batch holds at most 65535 members");
  for (int q = 0; q < count; q++) {
    if (!members[q]) return fail(FDTD_ERR_BADARG, "batch member %d is NULL", q);
    if (members[q]->device != members[0]->device || members[q]->prec != members[0]->prec)
      return fail(FDTD_ERR_BADARG, "batch member %d differs from member 0 in device or precision", q);
    for (int r = 0; r < q; r++)
      if (members[r] == members[q]) return fail(FDTD_ERR_BADARG, "batch member %d repeats member %d", q, r);
  }
  fdtd_batch* b = new fdtd_batch();
  b->device = members[0]->device;
  b->prec = members[0]->prec;
  b->m.assign(members, members + count);
  if (cudaSetDevice(b->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return fail(FDTD_ERR_CUDA, "cannot create a stream on device %d", members[0]->device);
  }
  BatchCtl zero{};
  if (cudaMalloc((void**)&b->d_ctl, sizeof(BatchCtl)) != cudaSuccess ||
      cudaMemcpyAsync(b->d_ctl, &zero, sizeof(BatchCtl), cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess) {
    fdtd_batch_free(b);
    return fail(FDTD_ERR_CUDA, "cannot allocate the batch control block");
  }
  *out = b;
  return FDTD_OK;
}

void fdtd_batch_free(fdtd_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop_graph(b);
  cudaFree(b->d_inst);
  cudaFree(b->d_tiles);
  cudaFree(b->d_mid);
  cudaFree(b->d_epi);
  cudaFree(b->d_flush);
  cudaFree(b->d_ctl);
  for (cudaStream_t st : b->ws) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (cudaEvent_t ev : b->wev) cudaEventDestroy(ev);
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int fdtd_batch_set_tiling(fdtd_batch* b, int x_planes_per_thread, int block_rows, int prefetch, int group) {
  if (!b) return fail(FDTD_ERR_BADARG, "NULL batch");
  if (x_planes_per_thread < 1 || x_planes_per_thread > 1024)
    return fail(FDTD_ERR_BADARG, "x planes per thread %d outside 1..1024", x_planes_per_thread);
  if (block_rows != 1 && block_rows != 2 && block_rows != 4 && block_rows != 8 && block_rows != 16)
    return fail(FDTD_ERR_BADARG, "block rows %d not in {1,2,4,8,16}", block_rows);
  if (prefetch < 1 || prefetch > 4) return fail(FDTD_ERR_BADARG, "prefetch depth %d not in 1..4", prefetch);
  if (prefetch > 2 && b->prec != FDTD_PREC_F32_TABLE)
    return fail(FDTD_ERR_BADARG, "prefetch depths 3 and 4 (shared-memory stages) need material-table members");
  if (group < 0 || group > 4096) return fail(FDTD_ERR_BADARG, "tile group %d outside 0..4096", group);
  if (b->ichunk != x_planes_per_thread || b->block_rows != block_rows || b->prefetch != prefetch ||
      b->group != group)
    batch_drop_graph(b);
  b->ichunk = x_planes_per_thread;
  b->block_rows = block_rows;
  b->prefetch = prefetch;
  b->group = group;
  return FDTD_OK;
}

int fdtd_batch_set_block_width(fdtd_batch* b, int threads_along_k) {
  if (!b) return fail(FDTD_ERR_BADARG, "NULL batch");
  if (threads_along_k != 16 && threads_along_k != 32)
    return fail(FDTD_ERR_BADARG, "block width %d not 16 or 32", threads_along_k);
  if (threads_along_k != b->block_w) batch_drop_graph(b);
  b->block_w = threads_along_k;
  return FDTD_OK;
}

int fdtd_batch_get_block_width(const fdtd_batch* b, int* threads_along_k) {
  if (!b || !threads_along_k) return fail(FDTD_ERR_BADARG, "NULL argument");
  *threads_along_k = b->block_w;
  return FDTD_OK;
}

int fdtd_batch_get_tiling(const fdtd_batch* b, int* x_planes_per_thread, int* block_rows, int* prefetch,
                          int* group) {
  if (!b || !x_planes_per_thread || !block_rows || !prefetch || !group) return fail(FDTD_ERR_BADARG, "NULL argument");
  *x_planes_per_thread = b->ichunk;
  *block_rows = b->block_rows;
  *prefetch = b->prefetch;
  *group = b->group;
  return FDTD_OK;
}

int fdtd_batch_set_streams(fdtd_batch* b, int streams) {
  if (!b) return fail(FDTD_ERR_BADARG, "NULL batch");
  if (streams < 0 || streams > kMaxBatchStreams)
    return fail(FDTD_ERR_BADARG, "worker streams %d outside 0..%d", streams, kMaxBatchStreams);
  if (streams != b->streams) batch_drop_graph(b);
  b->streams = streams;
  return FDTD_OK;
}

int fdtd_batch_set_members_per_launch(fdtd_batch* b, int members) {
  if (!b) return fail(FDTD_ERR_BADARG, "NULL batch");
  if (members < 0 || members > kGroupMembers)
    return fail(FDTD_ERR_BADARG, "members per launch %d outside 0..%d", members, kGroupMembers);
  if (members != b->members_per_launch) batch_drop_graph(b);
  b->members_per_launch = members;
  return FDTD_OK;
}

int fdtd_batch_get_members_per_launch(const fdtd_batch* b, int* members) {
  if (!b || !members) return fail(FDTD_ERR_BADARG, "NULL argument");
  *members = b->members_per_launch;
  return FDTD_OK;
}

int fdtd_batch_get_streams(const fdtd_batch* b, int* streams) {
  if (!b || !streams) return fail(FDTD_ERR_BADARG, "NULL argument");
  *streams = b->streams;
  return FDTD_OK;
}

int fdtd_batch_run(fdtd_batch* b, int count) {
  if (!b) return fail(FDTD_ERR_BADARG, "NULL batch");
  return batch_run(b, count);
}

int fdtd_batch_run_timed(fdtd_batch* b, int count, float* ms) {
  if (!b || !ms) return fail(FDTD_ERR_BADARG, "NULL argument");
  return batch_run(b, count, ms);
}

int fdtd_batch_profile_kernels(fdtd_batch* b, int count, double* avg_ms) {
  if (!b || !avg_ms || count < 1) return fail(FDTD_ERR_BADARG, "bad arguments");
  KernelTimer tm;
  CK(cudaSetDevice(b->device));
  for (int q = 0; q < 5; q++) CK(cudaEventCreate(&tm.ev[q]));
  int rc = batch_run(b, count, nullptr, &tm);
  for (int q = 0; q < 5; q++) cudaEventDestroy(tm.ev[q]);
  if (rc) return rc;
  for (int q = 0; q < 4; q++) avg_ms[q] = tm.ms[q] / count;
  return FDTD_OK;
}

int fdtd_batch_size(const fdtd_batch* b) { return b ? (int)b->m.size() : -1; }

// ===========================================================================
// Legacy global-context API (fdtd_cuda.h), FP32 per-cell coefficients.
// ===========================================================================
static fdtd_ctx* g_legacy = nullptr;

int fdtd_init(const FdtdDims* d) {
  if (!d) return fail(FDTD_ERR_BADARG, "NULL dims");
  fdtd_free(g_legacy);
  g_legacy = nullptr;
  FdtdConfig cfg{d->nx, d->ny, d->nz, d->dx, d->dy, d->dz, d->dt, d->numberOfTimeSteps, FDTD_PREC_F32, 0};
  return fdtd_create(&cfg, &g_legacy);
}

static std::vector<double> widen(const float* p, long long n) {
  std::vector<double> v(std::max<long long>(n, 0));
  for (long long q = 0; q < n; q++) v[q] = p[q];
  return v;
}

int fdtd_upload_coeff(int which, const float* host, int n) {
  if (!g_legacy) return fail(FDTD_ERR_STATE, "fdtd_init not called");
  if (!host) return fail(FDTD_ERR_BADARG, "NULL array");
  auto v = widen(host, n);
  return fdtd_ctx_upload_coeff(g_legacy, which, v.data(), n);
}

int fdtd_upload_cpml(int faceId, int nc, const float* b_e, const float* a_e, const float* b_m, const float* a_m,
                     const float* CPsi0, int n0, const float* CPsi1, int n1, const float* CPsi2, int n2,
                     const float* CPsi3, int n3, int m_start, int e_start, int ascending) {
  (void)ascending;  // the band starts carry the same information
  if (!g_legacy) return fail(FDTD_ERR_STATE, "fdtd_init not called");
  if (nc > 0 && (!b_e || !a_e || !b_m || !a_m)) return fail(FDTD_ERR_BADARG, "missing b/a profile");
  auto be = nc > 0 ? widen(b_e, nc) : std::vector<double>(), ae = nc > 0 ? widen(a_e, nc) : std::vector<double>();
  auto bm = nc > 0 ? widen(b_m, nc) : std::vector<double>(), am = nc > 0 ? widen(a_m, nc) : std::vector<double>();
  auto c0 = CPsi0 ? widen(CPsi0, n0) : std::vector<double>(), c1 = CPsi1 ? widen(CPsi1, n1) : std::vector<double>();
  auto c2 = CPsi2 ? widen(CPsi2, n2) : std::vector<double>(), c3 = CPsi3 ? widen(CPsi3, n3) : std::vector<double>();
  return fdtd_ctx_upload_cpml(g_legacy, faceId, nc, be.data(), ae.data(), bm.data(), am.data(), nullptr, nullptr,
                              CPsi0 ? c0.data() : nullptr, n0, CPsi1 ? c1.data() : nullptr, n1,
                              CPsi2 ? c2.data() : nullptr, n2, CPsi3 ? c3.data() : nullptr, n3, m_start, e_start);
}

int fdtd_upload_vsource(int dir, const int* idx, const float* coef, int count, const float* waveform, int nSteps) {
  if (!g_legacy) return fail(FDTD_ERR_STATE, "fdtd_init not called");
  if (!coef || !waveform) return fail(FDTD_ERR_BADARG, "NULL array");
  auto cs = widen(coef, count), wv = widen(waveform, nSteps);
  return fdtd_ctx_add_vsource(g_legacy, dir, idx, cs.data(), count, wv.data(), nSteps);
}

int fdtd_upload_svoltage(int dir, const int* idx, int count, float Csvf) {
  if (!g_legacy) return fail(FDTD_ERR_STATE, "fdtd_init not called");
  return fdtd_ctx_add_svoltage(g_legacy, dir, idx, count, Csvf);
}

int fdtd_upload_scurrent(const int* hxIdx, const float* hxW, int hxN, const int* hyIdx, const float* hyW, int hyN,
                         const int* hzIdx, const float* hzW, int hzN) {
  if (!g_legacy) return fail(FDTD_ERR_STATE, "fdtd_init not called");
  std::vector<int> comp, idx;
  std::vector<double> w;
  const int* I[3] = {hxIdx, hyIdx, hzIdx};
  const float* W[3] = {hxW, hyW, hzW};
  const int N[3] = {hxN, hyN, hzN};
  for (int c = 0; c < 3; c++) {
    if (N[c] > 0 && (!I[c] || !W[c])) return fail(FDTD_ERR_BADARG, "NULL gather list");
    for (int q = 0; q < N[c]; q++) {
      comp.push_back(c);
      idx.push_back(I[c][q]);
      w.push_back(W[c][q]);
    }
  }
  return fdtd_ctx_add_scurrent(g_legacy, comp.data(), idx.data(), w.data(), (int)comp.size());
}

int fdtd_run_batch(int tsStart, int count, float* svOut, float* siOut) {
  if (!g_legacy) return fail(FDTD_ERR_STATE, "fdtd_init not called");
  if (tsStart != g_legacy->ts) return fail(FDTD_ERR_BADARG, "batch starts at %d, the problem is at step %d", tsStart, g_legacy->ts);
  int rc = fdtd_ctx_run(g_legacy, count);
  if (rc && rc != FDTD_ERR_NONFINITE) return rc;
  std::vector<double> tmp(g_legacy->nsteps);
  if (svOut && !g_legacy->vprobe.empty()) {
    int r2 = fdtd_ctx_read_trace(g_legacy, 0, 0, tmp.data(), tsStart + count);
    if (r2) return r2;
    for (int q = 0; q < count; q++) svOut[q] = (float)tmp[tsStart + q];
  }
  if (siOut && !g_legacy->iprobe.empty()) {
    int r2 = fdtd_ctx_read_trace(g_legacy, 1, 0, tmp.data(), tsStart + count);
    if (r2) return r2;
    for (int q = 0; q < count; q++) siOut[q] = (float)tmp[tsStart + q];
  }
  return rc;
}

int fdtd_read_field(int which, float* host, int n) {
  if (!g_legacy) return fail(FDTD_ERR_STATE, "fdtd_init not called");
  if (!host) return fail(FDTD_ERR_BADARG, "NULL array");
  std::vector<double> tmp(std::max(n, 0));
  int rc = fdtd_ctx_read_field(g_legacy, which, tmp.data(), n);
  if (rc) return rc;
  for (int q = 0; q < n; q++) host[q] = (float)tmp[q];
  return FDTD_OK;
}

void fdtd_destroy(void) {
  fdtd_free(g_legacy);
  g_legacy = nullptr;
}

}  // extern "C"
