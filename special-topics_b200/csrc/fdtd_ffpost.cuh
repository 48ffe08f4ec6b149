// fdtd_ffpost.cuh -- far-field post-processing on the device: radiated power
// and directivity from the running NF-FF DFT accumulators
// (js_fdtd/src/farfield.js:257-607, restated in postproc.py for the host).
//
// Radiated power: per frequency, the surface integral of the Poynting flux
// of the equivalent currents, sum over faces and points of
// sign * area * (M1.J1 - M2.J2) / 2 (farfield.js:257-325).
//
// Directivity: for each frequency and direction (theta, phi), the radiation
// vectors N = sum J exp(jk r'.r) dA and L = sum M exp(jk r'.r) dA over the six
// faces, projected on theta/phi (farfield.js:328-607), then
// D_theta = k^2 |L_phi + eta N_theta|^2 / (8 pi eta P_rad), and D_phi alike
// with |L_theta - eta N_phi|^2.  Face points lie on a regular grid, so along
// the fastest-varying point index the phase factor advances by one complex
// multiply per point; one sincos starts each run of points.  Each block takes
// one frequency and 512 directions (two per thread), staging the face points'
// currents through shared memory so that every point is read once per block.
#pragma once
#include "fdtd_common.cuh"

namespace fdtd {

struct FFPost {
  const double* acc;
  long long off[24];
  long long sz[3];
  int nFreq;
  int ni, nj, nk;        // box extents in cells
  double pos0[3];        // first face point along x, y, z relative to the box centre
  double face[3][2];     // face planes (p, n) along x, y, z relative to the centre
  double d[3];           // cell sizes
};

constexpr double kC0 = 2.99792458e8;
constexpr double kEta0 = 376.73031346177066;
constexpr double kPi = 3.141592653589793;

// Accumulator names of face f (0..5 = xp xn yp yn zp zn): J1, J2, M1, M2.
__device__ __forceinline__ void face_arrays(int f, int& j1, int& j2, int& m1, int& m2) {
  static constexpr int tab[6][4] = {{CJYXP, CJZXP, CMYXP, CMZXP}, {CJYXN, CJZXN, CMYXN, CMZXN},
                                    {CJXYP, CJZYP, CMXYP, CMZYP}, {CJXYN, CJZYN, CMXYN, CMZYN},
                                    {CJXZP, CJYZP, CMXZP, CMYZP}, {CJXZN, CJYZN, CMXZN, CMYZN}};
  j1 = tab[f][0];
  j2 = tab[f][1];
  m1 = tab[f][2];
  m2 = tab[f][3];
}

// Compensated FP32 accumulator pairs (sum, compensation) -> FP64 values.
__global__ void k_kahan_to_f64(const double* __restrict__ acc, double* __restrict__ out, long long n) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float2 v = reinterpret_cast<const float2*>(acc)[q];
  out[q] = (double)v.x - (double)v.y;
}

// Radiated power of every frequency: block f, fixed-order reduction.
__global__ void __launch_bounds__(256) k_ff_power(FFPost P, double* __restrict__ radp) {
  __shared__ double red[256];
  const int f = blockIdx.x;
  double s = 0.0;
  // (face, area, M1, J1, M2, J2, sign) as farfield.js:257-325 pairs them
  const int terms[6][5] = {{CMYZP, CJXZP, CMXZP, CJYZP, 1},  {CMYZN, CJXZN, CMXZN, CJYZN, -1},
                           {CMXYP, CJZYP, CMZYP, CJXYP, 1},  {CMXYN, CJZYN, CMZYN, CJXYN, -1},
                           {CMZXP, CJYXP, CMYXP, CJZXP, 1},  {CMZXN, CJYXN, CMYXN, CJZXN, -1}};
  const int ax[6] = {2, 2, 1, 1, 0, 0};
  for (int t = 0; t < 6; t++) {
    const int a = ax[t];
    const long long n = P.sz[a];
    const double area = a == 0 ? P.d[1] * P.d[2] : a == 1 ? P.d[0] * P.d[2] : P.d[0] * P.d[1];
    const double* m1 = P.acc + P.off[terms[t][0]] + (long long)f * n;
    const double* j1 = P.acc + P.off[terms[t][1]] + (long long)f * n;
    const double* m2 = P.acc + P.off[terms[t][2]] + (long long)f * n;
    const double* j2 = P.acc + P.off[terms[t][3]] + (long long)f * n;
    const long long im = (long long)P.nFreq * n;  // imaginary parts follow the real ones
    double fs = 0.0;
    for (long long p = threadIdx.x; p < n; p += 256)
      fs += m1[p] * j1[p] + m1[p + im] * j1[p + im] - m2[p] * j2[p] - m2[p + im] * j2[p + im];
    s += terms[t][4] * area * fs;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) radp[f] = 0.5 * red[0];
}

struct Cplx {
  double re, im;
};
__device__ __forceinline__ Cplx cmul(Cplx a, Cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ void cmac(Cplx& s, Cplx e, double re, double im) {
  s.re += e.re * re - e.im * im;
  s.im += e.re * im + e.im * re;
}
__device__ __forceinline__ Cplx cexpj(double phase) {
  double s, c;
  sincos(phase, &s, &c);
  return {c, s};
}

constexpr int kFFAng = 2;  // directions per thread

__global__ void __launch_bounds__(256) k_ff_pattern(FFPost P, const double* __restrict__ freqs,
                                                    const double* __restrict__ theta, const double* __restrict__ phi,
                                                    int nang, const double* __restrict__ radp, double* __restrict__ dth,
                                                    double* __restrict__ dph) {
  __shared__ double sd[8][256];  // J1 J2 M1 M2 (re, im) of up to 256 points
  const int f = blockIdx.y;
  const double k = 2.0 * kPi * freqs[f] / kC0;
  double dir[kFFAng][3], st[kFFAng], ct[kFFAng], sp[kFFAng], cp[kFFAng];
  Cplx Nt[kFFAng], Np[kFFAng], Lt[kFFAng], Lp[kFFAng];
  for (int q = 0; q < kFFAng; q++) {
    const int a = (blockIdx.x * kFFAng + q) * 256 + threadIdx.x;
    const double th = a < nang ? theta[a] : 0.0, ph = a < nang ? phi[a] : 0.0;
    sincos(th, &st[q], &ct[q]);
    sincos(ph, &sp[q], &cp[q]);
    dir[q][0] = st[q] * cp[q];
    dir[q][1] = st[q] * sp[q];
    dir[q][2] = ct[q];
    Nt[q] = Np[q] = Lt[q] = Lp[q] = Cplx{0.0, 0.0};
  }
  const long long im_stride[3] = {(long long)P.nFreq * P.sz[0], (long long)P.nFreq * P.sz[1],
                                   (long long)P.nFreq * P.sz[2]};
  const int ext[3] = {P.ni, P.nj, P.nk};
  for (int fc = 0; fc < 6; fc++) {
    const int a = fc / 2, side = fc % 2;
    // point grid of the face: outer axis o, inner (fastest) axis n
    const int o = a == 0 ? 1 : 0, n = a == 2 ? 1 : 2;
    const int no = ext[o], nn = ext[n];
    int j1, j2, m1, m2;
    face_arrays(fc, j1, j2, m1, m2);
    const long long base = (long long)f * P.sz[a];
    Cplx S[kFFAng][4];
    Cplx step[kFFAng];
    for (int q = 0; q < kFFAng; q++) {
      for (int w = 0; w < 4; w++) S[q][w] = Cplx{0.0, 0.0};
      step[q] = cexpj(k * P.d[n] * dir[q][n]);
    }
    for (int r = 0; r < no; r++) {
      for (int c0 = 0; c0 < nn; c0 += 256) {
        const int cnt = min(256, nn - c0);
        __syncthreads();
        if (threadIdx.x < cnt) {
          const long long p = base + (long long)r * nn + c0 + threadIdx.x;
          const int arr[4] = {j1, j2, m1, m2};
          for (int w = 0; w < 4; w++) {
            const double* A = P.acc + P.off[arr[w]];
            sd[2 * w][threadIdx.x] = A[p];
            sd[2 * w + 1][threadIdx.x] = A[p + im_stride[a]];
          }
        }
        __syncthreads();
        for (int q = 0; q < kFFAng; q++) {
          const double ph0 = k * (P.face[a][side] * dir[q][a] + (P.pos0[o] + r * P.d[o]) * dir[q][o] +
                                  (P.pos0[n] + c0 * P.d[n]) * dir[q][n]);
          Cplx e = cexpj(ph0);
          for (int t = 0; t < cnt; t++) {
            for (int w = 0; w < 4; w++) cmac(S[q][w], e, sd[2 * w][t], sd[2 * w + 1][t]);
            e = cmul(e, step[q]);
          }
        }
      }
    }
    // project the face sums (farfield.js:328-607)
    const double A = a == 0 ? P.d[1] * P.d[2] : a == 1 ? P.d[0] * P.d[2] : P.d[0] * P.d[1];
    for (int q = 0; q < kFFAng; q++) {
      const Cplx J1 = S[q][0], J2 = S[q][1], M1 = S[q][2], M2 = S[q][3];
      double t1, t2, p1, p2;  // N_theta = t1 J1 + t2 J2, N_phi = p1 J1 + p2 J2 (same for L with M)
      if (a == 0) {           // J1 = Jy, J2 = Jz
        t1 = A * ct[q] * sp[q]; t2 = -A * st[q]; p1 = A * cp[q]; p2 = 0.0;
      } else if (a == 1) {    // J1 = Jx, J2 = Jz
        t1 = A * ct[q] * cp[q]; t2 = -A * st[q]; p1 = -A * sp[q]; p2 = 0.0;
      } else {                // J1 = Jx, J2 = Jy
        t1 = A * ct[q] * cp[q]; t2 = A * ct[q] * sp[q]; p1 = -A * sp[q]; p2 = A * cp[q];
      }
      Nt[q].re += t1 * J1.re + t2 * J2.re;
      Nt[q].im += t1 * J1.im + t2 * J2.im;
      Np[q].re += p1 * J1.re + p2 * J2.re;
      Np[q].im += p1 * J1.im + p2 * J2.im;
      Lt[q].re += t1 * M1.re + t2 * M2.re;
      Lt[q].im += t1 * M1.im + t2 * M2.im;
      Lp[q].re += p1 * M1.re + p2 * M2.re;
      Lp[q].im += p1 * M1.im + p2 * M2.im;
    }
  }
  const double scale = k * k / (8.0 * kPi * kEta0 * radp[f]);
  for (int q = 0; q < kFFAng; q++) {
    const int a = (blockIdx.x * kFFAng + q) * 256 + threadIdx.x;
    if (a >= nang) continue;
    const double ar = Lp[q].re + kEta0 * Nt[q].re, ai = Lp[q].im + kEta0 * Nt[q].im;
    const double br = Lt[q].re - kEta0 * Np[q].re, bi = Lt[q].im - kEta0 * Np[q].im;
    dth[(long long)f * nang + a] = scale * (ar * ar + ai * ai);
    dph[(long long)f * nang + a] = scale * (br * br + bi * bi);
  }
}

}  // namespace fdtd
