// fdtd_common.cuh -- shared device types and the per-step epilogue (port
// voltages + running far-field DFT) used by every field layout.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fdtd {

constexpr int kMaxSources = 8;
constexpr int kMaxProbes = 8;

// Exactly rounded arithmetic that nvcc may not contract into FMA.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

struct GridDims {
  int nx, ny, nz;
};

template <typename T>
struct Fields {
  T *Hx, *Hy, *Hz, *Ex, *Ey, *Ez;
};

// One CPML face.  Psi slots: x face 0=hyx 1=hzx 2=eyx 3=ezx; y face 0=hxy 1=hzy
// 2=ezy 3=exy; z face 0=hxz 1=hyz 2=exz 3=eyz (js_fdtd/src/cpml.js:147-448).
template <typename T>
struct Face {
  int nc;       // 0 when the face is not a CPML
  int m_start;  // first H index of the band along the face axis
  int e_start;  // first E index of the band along the face axis
  const T *b_e, *a_e, *b_m, *a_m;
  const float *inv_ke, *inv_km;  // 1/kappa per band cell (material-table problems only)
  T* psi[4];
  const T* cpsi[4];
};

struct SourceBox {
  int comp;                    // 0=Ex 1=Ey 2=Ez
  int i0, i1, j0, j1, k0, k1;  // inclusive component-index box
};

template <typename T>
struct Sources {
  int n;
  SourceBox box[kMaxSources];
  const T* cs[kMaxSources];    // per-cell source coefficient (Cexs / Ceys / Cezs)
  const T* wave[kMaxSources];  // voltage_per_e_field, one value per step
};

struct Probes {
  int n_v, n_i;
  int v_comp[kMaxProbes];
  int v_count[kMaxProbes];
  const int* v_idx[kMaxProbes];
  double v_csvf[kMaxProbes];
  int i_count[kMaxProbes];
  const int* i_comp[kMaxProbes];
  const int* i_idx[kMaxProbes];
  const double* i_w[kMaxProbes];
  double* V;   // [n_v][nsteps]
  double* I;   // [n_i][nsteps]
  int nsteps;
  int* status; // [0] = watchdog code, [1] = first non-finite step
};

struct FarField {
  int nFreq;
  int LI, LJ, LK, UI, UJ, UK;  // 0-based box planes
  int ni, nj, nk;              // box extents in cells
  const double* ph;            // [nsteps][nFreq][4] = cos_h, -sin_h, cos_e, -sin_e
  double* acc;                 // 24 arrays, each re[nFreq][sz] then im[nFreq][sz]
  long long off[24];
  long long sz[3];             // x-, y-, z-face point counts
  int kahan;                   // accumulators are FP32 (sum, compensation) pairs, not FP64
  int block;                   // > 0: steps per time block (samples buffered, accumulated by k_dft_flush)
  float* samples;              // [block][points][8] surface samples of the open block
  const int* done;             // steps already accumulated
};



// Lumped source on the cell this thread owns (sources.js:271-288).
template <typename T>
__device__ __forceinline__ void inject_sources(const Sources<T>& s, int comp, int i, int j, int k, int ts, T& e) {
  for (int q = 0; q < s.n; q++) {
    const SourceBox& b = s.box[q];
    if (b.comp == comp && i >= b.i0 && i <= b.i1 && j >= b.j0 && j <= b.j1 && k >= b.k0 && k <= b.k1) {
      const int ni = b.i1 - b.i0 + 1, nj = b.j1 - b.j0 + 1;
      const int n = ((k - b.k0) * nj + (j - b.j0)) * ni + (i - b.i0);
      e = add(e, mul(s.cs[q][n], s.wave[q][ts]));
    }
  }
}

template <typename T>
__device__ __forceinline__ const T* comp_ptr(const Fields<T>& f, int c) {
  return c == 0 ? f.Hx : c == 1 ? f.Hy : c == 2 ? f.Hz : c == 3 ? f.Ex : c == 4 ? f.Ey : f.Ez;
}

// Port current: ordered weighted sum of H samples (sampling.js:204-245).
template <typename T>
__device__ void current_probe(const Fields<T>& f, const Probes& pr, int q, int ts) {
  double sv = 0.0;
  const int n = pr.i_count[q];
  for (int m = 0; m < n; m++) {
    const double h = (double)comp_ptr(f, pr.i_comp[q][m])[pr.i_idx[q][m]];
    sv = add(sv, mul(pr.i_w[q][m], h));
  }
  pr.I[(long long)q * pr.nsteps + ts] = sv;
}

// Port voltage: V = Csvf * (sequential sum of the gap samples) (sampling.js:295-307).
template <typename T>
__device__ void voltage_probe(const Fields<T>& f, const Probes& pr, int q, int ts) {
  const T* F = comp_ptr(f, 3 + pr.v_comp[q]);
  double sum = 0.0;
  const int n = pr.v_count[q];
  for (int m = 0; m < n; m++) sum = add(sum, (double)F[pr.v_idx[q][m]]);
  const double v = mul(pr.v_csvf[q], sum);
  pr.V[(long long)q * pr.nsteps + ts] = v;
  if (!isfinite(v)) {
    atomicExch(&pr.status[0], 5);
    atomicMin(&pr.status[1], ts);
  }
}

// Names of the 24 accumulator arrays, in FarField::off order.
enum {
  CJYXP, CJZXP, CJYXN, CJZXN, CJXYP, CJZYP, CJXYN, CJZYN, CJXZP, CJYZP, CJXZN, CJYZN,
  CMYXP, CMZXP, CMYXN, CMZXN, CMXYP, CMZYP, CMXYN, CMZYN, CMXZP, CMYZP, CMXZN, CMYZN
};

// The 8 accumulator arrays a surface point feeds, in sample order, for the
// x-face (0), y-face (1) and z-face (2) point pairs.
__device__ __forceinline__ int sample_array(int group, int a) {
  static constexpr int tab[3][8] = {{CMYXP, CMZXP, CJYXP, CJZXP, CMYXN, CMZXN, CJYXN, CJZXN},
                                    {CMXYP, CMZYP, CJZYP, CJXYP, CMXYN, CMZYN, CJZYN, CJXYN},
                                    {CMXZP, CMYZP, CJXZP, CJYZP, CMXZN, CMYZN, CJXZN, CJYZN}};
  return tab[group][a];
}

// Time-blocked DFT: the epilogue stores a step's 8 samples per point in slot
// ts % block; this writes them into the running accumulators.
__device__ __forceinline__ void store_samples(const FarField& ff, long long t, int ts, const double* v) {
  const long long npts = ff.sz[0] + ff.sz[1] + ff.sz[2];
  float* s = ff.samples + ((long long)(ts % ff.block) * npts + t) * 8;
#pragma unroll
  for (int a = 0; a < 8; a++) s[a] = (float)v[a];
}

// One Kahan-compensated FP32 step: v = (sum, compensation), sum += x.
__device__ __forceinline__ void kahan_add(float2* v, float x) {
  float2 a = *v;
  const float y = __fsub_rn(x, a.y);
  const float t = __fadd_rn(a.x, y);
  a.y = __fsub_rn(__fsub_rn(t, a.x), y);
  a.x = t;
  *v = a;
}

__device__ __forceinline__ void acc2(const FarField& ff, int a, long long p, double c, double s, double t) {
  double* re = ff.acc + ff.off[a] + p;
  double* im = re + ff.nFreq * ff.sz[(a % 12) / 4];
  if (ff.kahan) {
    const float tf = (float)t;
    kahan_add(reinterpret_cast<float2*>(re), __fmul_rn((float)c, tf));
    kahan_add(reinterpret_cast<float2*>(im), __fmul_rn((float)s, tf));
    return;
  }
  *re = add(*re, mul(c, t));
  *im = add(*im, mul(s, t));
}

// ---------------------------------------------------------------------------
// Epilogue: running NF-FF DFT (farfield.js:90-248) on the six Huygens faces,
// then the port voltages.  One thread per surface point (xp/xn, yp/yn and zp/zn
// pairs share the point), looping over frequencies.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void epilogue_thread(const Fields<T>& f, const GridDims& g, const FarField& ff,
                                                const Probes& probes, const int* ts_ptr, long long t) {
  const int ts = *ts_ptr;
  const int ny = g.ny, nz = g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const long long nff = ff.nFreq > 0 ? ff.sz[0] + ff.sz[1] + ff.sz[2] : 0;
  if (t >= nff) {
    const long long q = t - nff;
    if (q < probes.n_v) voltage_probe(f, probes, (int)q, ts);
    return;
  }
#define HX(i, j, k) (double)f.Hx[((long long)(i) * ny + (j)) * nz + (k)]
#define HY(i, j, k) (double)f.Hy[((long long)(i) * nyp1 + (j)) * nz + (k)]
#define HZ(i, j, k) (double)f.Hz[((long long)(i) * ny + (j)) * nzp1 + (k)]
#define EX(i, j, k) (double)f.Ex[((long long)(i) * nyp1 + (j)) * nzp1 + (k)]
#define EY(i, j, k) (double)f.Ey[((long long)(i) * ny + (j)) * nzp1 + (k)]
#define EZ(i, j, k) (double)f.Ez[((long long)(i) * nyp1 + (j)) * nz + (k)]
  const double* ph = ff.ph + (long long)ts * ff.nFreq * 4;
  if (t < ff.sz[0]) {
    const int nj = (int)(t / ff.nk), nk = (int)(t % ff.nk);
    const int j0 = ff.LJ + nj, k0 = ff.LK + nk, UI = ff.UI, LI = ff.LI;
    const double tmyxp = mul(0.5, add(EZ(UI, j0, k0), EZ(UI, j0 + 1, k0)));
    const double tmzxp = mul(-0.5, add(EY(UI, j0, k0), EY(UI, j0, k0 + 1)));
    const double tjyxp = mul(-0.25, add(add(add(HZ(UI, j0, k0), HZ(UI, j0, k0 + 1)), HZ(UI - 1, j0, k0)), HZ(UI - 1, j0, k0 + 1)));
    const double tjzxp = mul(0.25, add(add(add(HY(UI, j0, k0), HY(UI, j0 + 1, k0)), HY(UI - 1, j0, k0)), HY(UI - 1, j0 + 1, k0)));
    const double tmyxn = mul(-0.5, add(EZ(LI, j0, k0), EZ(LI, j0 + 1, k0)));
    const double tmzxn = mul(0.5, add(EY(LI, j0, k0), EY(LI, j0, k0 + 1)));
    const double tjyxn = mul(0.25, add(add(add(HZ(LI, j0, k0), HZ(LI, j0, k0 + 1)), HZ(LI - 1, j0, k0)), HZ(LI - 1, j0, k0 + 1)));
    const double tjzxn = mul(-0.25, add(add(add(HY(LI, j0, k0), HY(LI, j0 + 1, k0)), HY(LI - 1, j0, k0)), HY(LI - 1, j0 + 1, k0)));
    if (ff.block) {  // time-blocked: buffer the samples, k_dft_flush accumulates them
      const double v[8] = {tmyxp, tmzxp, tjyxp, tjzxp, tmyxn, tmzxn, tjyxn, tjzxn};
      store_samples(ff, t, ts, v);
      return;
    }
    for (int m = 0; m < ff.nFreq; m++) {
      const long long p = (long long)m * ff.sz[0] + t;
      const double ch = ph[4 * m], sh = ph[4 * m + 1], ce = ph[4 * m + 2], se = ph[4 * m + 3];
      acc2(ff, CMYXP, p, ce, se, tmyxp);
      acc2(ff, CMZXP, p, ce, se, tmzxp);
      acc2(ff, CJYXP, p, ch, sh, tjyxp);
      acc2(ff, CJZXP, p, ch, sh, tjzxp);
      acc2(ff, CMYXN, p, ce, se, tmyxn);
      acc2(ff, CMZXN, p, ce, se, tmzxn);
      acc2(ff, CJYXN, p, ch, sh, tjyxn);
      acc2(ff, CJZXN, p, ch, sh, tjzxn);
    }
  } else if (t < ff.sz[0] + ff.sz[1]) {
    const long long q = t - ff.sz[0];
    const int ni = (int)(q / ff.nk), nk = (int)(q % ff.nk);
    const int i0 = ff.LI + ni, k0 = ff.LK + nk, UJ = ff.UJ, LJ = ff.LJ;
    const double tmxyp = mul(-0.5, add(EZ(i0, UJ, k0), EZ(i0 + 1, UJ, k0)));
    const double tmzyp = mul(0.5, add(EX(i0, UJ, k0), EX(i0, UJ, k0 + 1)));
    const double tjzyp = mul(-0.25, add(add(add(HX(i0, UJ, k0), HX(i0 + 1, UJ, k0)), HX(i0, UJ - 1, k0)), HX(i0 + 1, UJ - 1, k0)));
    const double tjxyp = mul(0.25, add(add(add(HZ(i0, UJ, k0), HZ(i0, UJ, k0 + 1)), HZ(i0, UJ - 1, k0)), HZ(i0, UJ - 1, k0 + 1)));
    const double tmxyn = mul(0.5, add(EZ(i0, LJ, k0), EZ(i0 + 1, LJ, k0)));
    const double tmzyn = mul(-0.5, add(EX(i0, LJ, k0), EX(i0, LJ, k0 + 1)));
    const double tjzyn = mul(0.25, add(add(add(HX(i0, LJ, k0), HX(i0 + 1, LJ, k0)), HX(i0, LJ - 1, k0)), HX(i0 + 1, LJ - 1, k0)));
    const double tjxyn = mul(-0.25, add(add(add(HZ(i0, LJ, k0), HZ(i0, LJ, k0 + 1)), HZ(i0, LJ - 1, k0)), HZ(i0, LJ - 1, k0 + 1)));
    if (ff.block) {  // time-blocked: buffer the samples, k_dft_flush accumulates them
      const double v[8] = {tmxyp, tmzyp, tjzyp, tjxyp, tmxyn, tmzyn, tjzyn, tjxyn};
      store_samples(ff, t, ts, v);
      return;
    }
    for (int m = 0; m < ff.nFreq; m++) {
      const long long p = (long long)m * ff.sz[1] + q;
      const double ch = ph[4 * m], sh = ph[4 * m + 1], ce = ph[4 * m + 2], se = ph[4 * m + 3];
      acc2(ff, CMXYP, p, ce, se, tmxyp);
      acc2(ff, CMZYP, p, ce, se, tmzyp);
      acc2(ff, CJZYP, p, ch, sh, tjzyp);
      acc2(ff, CJXYP, p, ch, sh, tjxyp);
      acc2(ff, CMXYN, p, ce, se, tmxyn);
      acc2(ff, CMZYN, p, ce, se, tmzyn);
      acc2(ff, CJZYN, p, ch, sh, tjzyn);
      acc2(ff, CJXYN, p, ch, sh, tjxyn);
    }
  } else {
    const long long q = t - ff.sz[0] - ff.sz[1];
    const int ni = (int)(q / ff.nj), nj = (int)(q % ff.nj);
    const int i0 = ff.LI + ni, j0 = ff.LJ + nj, UK = ff.UK, LK = ff.LK;
    const double tmxzp = mul(0.5, add(EY(i0, j0, UK), EY(i0 + 1, j0, UK)));
    const double tmyzp = mul(-0.5, add(EX(i0, j0, UK), EX(i0, j0 + 1, UK)));
    const double tjxzp = mul(0.25, add(add(add(HX(i0, j0, UK), HX(i0 + 1, j0, UK)), HX(i0, j0, UK - 1)), HX(i0 + 1, j0, UK - 1)));
    const double tjxzp2 = mul(-0.25, add(add(add(HY(i0, j0, UK), HY(i0, j0 + 1, UK)), HY(i0, j0, UK - 1)), HY(i0, j0 + 1, UK - 1)));
    const double tmxzn = mul(-0.5, add(EY(i0, j0, LK), EY(i0 + 1, j0, LK)));
    const double tmyzn = mul(0.5, add(EX(i0, j0, LK), EX(i0, j0 + 1, LK)));
    const double tjxzn = mul(0.25, add(add(add(HY(i0, j0, LK), HY(i0, j0 + 1, LK)), HY(i0, j0, LK - 1)), HY(i0, j0 + 1, LK - 1)));
    const double tjyzn = mul(-0.25, add(add(add(HX(i0, j0, LK), HX(i0 + 1, j0, LK)), HX(i0, j0, LK - 1)), HX(i0 + 1, j0, LK - 1)));
    if (ff.block) {  // time-blocked: buffer the samples, k_dft_flush accumulates them
      const double v[8] = {tmxzp, tmyzp, tjxzp2, tjxzp, tmxzn, tmyzn, tjxzn, tjyzn};
      store_samples(ff, t, ts, v);
      return;
    }
    for (int m = 0; m < ff.nFreq; m++) {
      const long long p = (long long)m * ff.sz[2] + q;
      const double ch = ph[4 * m], sh = ph[4 * m + 1], ce = ph[4 * m + 2], se = ph[4 * m + 3];
      acc2(ff, CMXZP, p, ce, se, tmxzp);
      acc2(ff, CMYZP, p, ce, se, tmyzp);
      // zp Jx: the reference adds the Hx average, then swaps it for the Hy
      // average in a second statement (farfield.js:211-225); keep both roundings
      // (with compensated FP32 accumulators only the net Hy term is added).
      if (ff.kahan) {
        acc2(ff, CJXZP, p, ch, sh, tjxzp2);
      } else {
        double* re = ff.acc + ff.off[CJXZP] + p;
        double* im = re + ff.nFreq * ff.sz[2];
        const double r1 = add(*re, mul(ch, tjxzp));
        const double i1 = add(*im, mul(sh, tjxzp));
        *re = add(sub(r1, mul(ch, tjxzp)), mul(ch, tjxzp2));
        *im = add(sub(i1, mul(sh, tjxzp)), mul(sh, tjxzp2));
      }
      acc2(ff, CJYZP, p, ch, sh, tjxzp);  // the reference's zp Jy is the same Hx average
      acc2(ff, CMXZN, p, ce, se, tmxzn);
      acc2(ff, CMYZN, p, ce, se, tmyzn);
      acc2(ff, CJXZN, p, ch, sh, tjxzn);
      acc2(ff, CJYZN, p, ch, sh, tjyzn);
    }
  }
#undef HX
#undef HY
#undef HZ
#undef EX
#undef EY
#undef EZ
}

template <typename T>
__global__ void __launch_bounds__(256) k_epilogue(Fields<T> f, GridDims g, FarField ff, Probes probes,
                                                  const int* ts_ptr) {
  epilogue_thread<T>(f, g, ff, probes, ts_ptr, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Accumulates the buffered samples of steps [*ff.done, upto) into the
// running DFT: one thread per (surface point pair, frequency), steps in
// order.  upto < 0: flush only when the step just finished closes a block
// (upto = ts + 1 then), so the launch can sit in every step of a graph.
__device__ __forceinline__ void dft_flush_thread(const FarField& ff, const int* ts_ptr, int upto, long long q) {
  const long long npts = ff.sz[0] + ff.sz[1] + ff.sz[2];
  if (ff.block <= 0 || q >= npts * ff.nFreq) return;
  if (upto >= 0 && upto % ff.block == 0) return;  // closed by the flush inside its last step
  if (upto < 0) {
    const int ts = *ts_ptr;
    if ((ts + 1) % ff.block != 0) return;
    upto = ts + 1;
  }
  const int from = *ff.done;
  const long long t = q % npts;
  const int m = (int)(q / npts);
  const int group = t < ff.sz[0] ? 0 : t < ff.sz[0] + ff.sz[1] ? 1 : 2;
  const long long p = (long long)m * ff.sz[group] + (group == 0 ? t : group == 1 ? t - ff.sz[0] : t - ff.sz[0] - ff.sz[1]);
  for (int a = 0; a < 8; a++) {
    const int arr = sample_array(group, a);
    const int e = arr >= CMYXP ? 2 : 0;  // magnetic currents take the E-time phasor
    double* re = ff.acc + ff.off[arr] + p;
    double* im = re + ff.nFreq * ff.sz[group];
    if (ff.kahan) {
      for (int s = from; s < upto; s++) {
        const double* ph = ff.ph + ((long long)s * ff.nFreq + m) * 4 + e;
        const float v = ff.samples[((long long)(s % ff.block) * npts + t) * 8 + a];
        kahan_add(reinterpret_cast<float2*>(re), __fmul_rn((float)ph[0], v));
        kahan_add(reinterpret_cast<float2*>(im), __fmul_rn((float)ph[1], v));
      }
    } else {
      double r = *re, i = *im;
      for (int s = from; s < upto; s++) {
        const double* ph = ff.ph + ((long long)s * ff.nFreq + m) * 4 + e;
        const double v = ff.samples[((long long)(s % ff.block) * npts + t) * 8 + a];
        r += ph[0] * v;
        i += ph[1] * v;
      }
      *re = r;
      *im = i;
    }
  }
}

__global__ void __launch_bounds__(256) k_dft_flush(FarField ff, const int* ts_ptr, int upto) {
  dft_flush_thread(ff, ts_ptr, upto, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

}  // namespace fdtd
