// fdtd_step.cuh -- the FDTD half-step kernels for sm_100a.
//
// Per step (js_fdtd/src/backends/CONTRACT.md:61-96):
//   k_step_h    bulk H (fdtd_kernels.ts:20-114) fused with the magnetic CPML
//               Psi update and correction of all six faces (cpml.js:456-724)
//   k_step_mid  port currents (sampling.js:204-245) and the Ex(i=0) plane that
//               the reference's Ey(i=nx) update reads through an out-of-range
//               Hz index (fdtd_kernels.ts:159-178)
//   k_step_e    bulk E (fdtd_kernels.ts:116-210) fused with the electric CPML
//               (cpml.js:727-1003) and lumped-source injection (sources.js:271-288)
//   k_epilogue  (fdtd_common.cuh) port voltages and the running NF-FF DFT
//
// Work split: a thread owns one (j,k) column of the (nx+1, ny+1, nz+1) box and
// walks a chunk of x planes, updating at every (i,j,k) the components that
// exist there.  Every field value and Psi element has exactly one writer, the
// x-neighbour of the previous plane is carried in a register (E(i+1) becomes
// E(i) for the H update, H(i) becomes H(i-1) for the E update), everything
// that depends only on (j,k) -- 32-bit offsets, y/z CPML band membership, the
// y/z 1/kappa factors, source-column hits -- is computed once per thread, and
// the CPML corrections of a value are applied in registers in the reference's
// face order xn xp yn yp zn zp right after its bulk update.
//
// Generic over how a cell finds its coefficients:
//   ArrayCoef<T>  the reference's 18 per-cell arrays (FP64 drop-in, FP32 legacy)
//   TableCoef     one uint8 material id per cell and component into a table of
//                 (self, curl1, curl2) rows without kappa; 1/kappa comes from 1-D
//                 per-axis profiles and CPsi = curl coefficient x cell size
// and over the arithmetic: EXACT uses the _rn intrinsics so nvcc never fuses a
// multiply into an add and every value sees the reference's sequence of
// rounded operations; otherwise FMA is allowed.
#pragma once
#include "fdtd_common.cuh"

namespace fdtd {

// ---------------------------------------------------------------------------
// Arithmetic policies
// ---------------------------------------------------------------------------
template <typename T, bool EXACT>
struct Ar;
template <typename T>
struct Ar<T, true> {
  static __device__ __forceinline__ T lin3(T c0, T h, T c1, T d1, T c2, T d2) {
    return add(add(mul(c0, h), mul(c1, d1)), mul(c2, d2));
  }
  static __device__ __forceinline__ T lin2(T b, T p, T a, T d) { return add(mul(b, p), mul(a, d)); }
  static __device__ __forceinline__ T axpy(T y, T c, T p) { return add(y, mul(c, p)); }
  static __device__ __forceinline__ T dif(T a, T b) { return sub(a, b); }
};
template <typename T>
struct Ar<T, false> {
  static __device__ __forceinline__ T lin3(T c0, T h, T c1, T d1, T c2, T d2) {
    return fma(c2, d2, fma(c1, d1, c0 * h));
  }
  static __device__ __forceinline__ T lin2(T b, T p, T a, T d) { return fma(a, d, b * p); }
  static __device__ __forceinline__ T axpy(T y, T c, T p) { return fma(c, p, y); }
  static __device__ __forceinline__ T dif(T a, T b) { return a - b; }
};

// ---------------------------------------------------------------------------
// Coefficient policies.  Component ids follow the field order 0..5 = Hx Hy Hz
// Ex Ey Ez.  For each component the two curl terms are
//   Hx: c1 Chxey dEy/dz (z faces)  c2 Chxez dEz/dy (y faces)
//   Hy: c1 Chyez dEz/dx (x faces)  c2 Chyex dEx/dz (z faces)
//   Hz: c1 Chzex dEx/dy (y faces)  c2 Chzey dEy/dx (x faces)
//   Ex: c1 Cexhz dHz/dy (y faces)  c2 Cexhy dHy/dz (z faces)
//   Ey: c1 Ceyhx dHx/dz (z faces)  c2 Ceyhz dHz/dx (x faces)
//   Ez: c1 Cezhy dHy/dx (x faces)  c2 Cezhx dHx/dy (y faces)
// get(): c0, c1, c2 as used by the update (kappa applied), u1, u2 without kappa.
// ---------------------------------------------------------------------------
template <typename T>
struct ArrayCoef {
  static constexpr bool kTable = false;
  const T* c[6][3];  // [component][self, curl1, curl2]
  __device__ __forceinline__ void get(int comp, int idx, float, float, T& c0, T& c1, T& c2, T& u1, T& u2) const {
    c0 = c[comp][0][idx];
    c1 = c[comp][1][idx];
    c2 = c[comp][2][idx];
    u1 = c1;
    u2 = c2;
  }
  __device__ __forceinline__ T cpsi(const Face<T>& F, int slot, int pi, T, T) const { return F.cpsi[slot][pi]; }
  __device__ __forceinline__ float invk(int, int) const { return 1.f; }
  // interior (kappa = 1) form split into the load and its use, for prefetching
  struct Raw {
    T a, b, c;
  };
  __device__ __forceinline__ Raw fetch(int comp, int idx) const {
    return Raw{c[comp][0][idx], c[comp][1][idx], c[comp][2][idx]};
  }
  __device__ __forceinline__ void decode(int, const Raw& r, T& c0, T& c1, T& c2) const {
    c0 = r.a;
    c1 = r.b;
    c2 = r.c;
  }
  // get() split into the load (fetch) and this: kappa is in the arrays already
  __device__ __forceinline__ void decode_k(int comp, const Raw& r, float, float, T& c0, T& c1, T& c2, T& u1,
                                           T& u2) const {
    decode(comp, r, c0, c1, c2);
    u1 = c1;
    u2 = c2;
  }
  // cpsi() split into a load that can be issued early and its use
  __device__ __forceinline__ T cpsi_fetch(const Face<T>& F, int slot, int pi) const { return F.cpsi[slot][pi]; }
  __device__ __forceinline__ T cpsi_use(T fetched, T, T) const { return fetched; }
};

constexpr int kTableRows = 256;

struct TableCoef {
  static constexpr bool kTable = true;
  const unsigned char* ids[6];  // per component, field order
  const float4* tab;            // [6][kTableRows] (self, curl1, curl2, 0) without kappa
  const float* inv[6];          // 1/kappa along x y z for E (0..2) and H (3..5), length n+1
  __device__ __forceinline__ void get(int comp, int idx, float k1, float k2, float& c0, float& c1, float& c2,
                                      float& u1, float& u2) const {
    const int id = __ldg(ids[comp] + idx);
    const float4 r = __ldg(tab + comp * kTableRows + id);
    c0 = r.x;
    u1 = r.y;
    u2 = r.z;
    c1 = u1 * k1;
    c2 = u2 * k2;
  }
  __device__ __forceinline__ float cpsi(const Face<float>&, int, int, float u, float dcell) const { return u * dcell; }
  // 1/kappa of E (h=0) or H (h=1) at position pos along axis a
  __device__ __forceinline__ float invk(int ha, int pos) const { return __ldg(inv[ha] + pos); }
  // interior (kappa = 1) form split into the id load and the row lookup
  using Raw = unsigned char;
  __device__ __forceinline__ Raw fetch(int comp, int idx) const { return __ldg(ids[comp] + idx); }
  __device__ __forceinline__ void decode(int comp, Raw id, float& c0, float& c1, float& c2) const {
    const float4 r = __ldg(tab + comp * kTableRows + id);
    c0 = r.x;
    c1 = r.y;
    c2 = r.z;
  }
  // get() split into the id load (fetch) and this row lookup with kappa
  __device__ __forceinline__ void decode_k(int comp, Raw id, float k1, float k2, float& c0, float& c1, float& c2,
                                           float& u1, float& u2) const {
    decode(comp, id, c0, u1, u2);
    c1 = u1 * k1;
    c2 = u2 * k2;
  }
  __device__ __forceinline__ float cpsi_fetch(const Face<float>&, int, int) const { return 0.f; }
  __device__ __forceinline__ float cpsi_use(float, float u, float dcell) const { return u * dcell; }
};

template <typename T, class C>
struct StepParams {
  GridDims g;
  Fields<T> f;
  C coef;
  Face<T> face[6];
  T* ex0b;   // scratch plane (ny x (nz+1)): Ex(i=0) after its bulk update
  int* ts;   // device step counter (index of the step being computed)
  Sources<T> src;
  T dcell[3];
  int ichunk;  // x planes per thread
  int bands_disjoint;  // per axis, no position lies in both CPML bands (H and E)
  int dft_block;       // time-blocked surface DFT: steps per block (0: per step)
  int* dft_done;       // steps the blocked DFT has accumulated
  // 0: Ey and Ez at i = nx are bulk-updated from the values the reference
  // reads one plane past Hz and Hy (fdtd_kernels.ts:159-204); 1: they are not
  // updated and stay zero, the ranges of the MATLAB original
  // (fdtd_solve_Ch9_ex9a_12032026.m.txt:2095-2106), a PEC wall.
  int x_wall;
  int* fault;   // the handle's status code word: 4 when a bounded wait of the bulk-staged form ran out
};

// Band of a face that contains `pos` (H: m band, E: e band): ci or -1.
template <typename T>
__device__ __forceinline__ int band_ci(const Face<T>& F, int pos, bool electric) {
  const int st = electric ? F.e_start : F.m_start;
  return (F.nc > 0 && pos >= st && pos < st + F.nc) ? pos - st : -1;
}

// One face's CPML on a value: Psi = b Psi + a drive, then v += CPsi Psi.
template <typename T, class C, bool EXACT, bool ELECTRIC>
__device__ __forceinline__ void cpml_apply(const C& coef, const Face<T>& F, int ci, int pi, int slot, T drive, T u,
                                           T dcell, T& v) {
  T* P = F.psi[slot];
  const T b = ELECTRIC ? F.b_e[ci] : F.b_m[ci];
  const T a = ELECTRIC ? F.a_e[ci] : F.a_m[ci];
  const T ps = Ar<T, EXACT>::lin2(b, P[pi], a, drive);
  P[pi] = ps;
  v = Ar<T, EXACT>::axpy(v, coef.cpsi(F, slot, pi, u, dcell), ps);
}

// The same correction as cpml_apply with Psi (and CPsi, per-cell layouts)
// loaded earlier and the band cell's profile values b and a held in
// registers: Psi = b Psi + a drive is stored at P, then v += CPsi Psi.
template <typename T, class C, bool EXACT>
__device__ __forceinline__ void cpml_fold(const C& coef, T* P, T b, T a, T psi, T cp, T drive, T u, T dcell, T& v) {
  const T ps = Ar<T, EXACT>::lin2(b, psi, a, drive);
  *P = ps;
  v = Ar<T, EXACT>::axpy(v, coef.cpsi_use(cp, u, dcell), ps);
}

// Profile values b, a of band cell ci of face f (H: m profiles, E: e
// profiles); zero when f < 0.
template <typename T, bool ELECTRIC>
__device__ __forceinline__ void band_profile(const Face<T>* face, int f, int ci, T& b, T& a) {
  b = T(0);
  a = T(0);
  if (f < 0) return;
  const Face<T>& F = face[f];
  b = __ldg((ELECTRIC ? F.b_e : F.b_m) + ci);
  a = __ldg((ELECTRIC ? F.a_e : F.a_m) + ci);
}

// Face of axis `a` (0..2) whose band holds `pos`, and the band cell; -1 if none.
// Only meaningful when the two bands of the axis are disjoint.
template <typename T>
__device__ __forceinline__ int band_face(const Face<T>* face, int a, int pos, bool electric, int& ci) {
  ci = band_ci(face[2 * a], pos, electric);
  if (ci >= 0) return 2 * a;
  ci = band_ci(face[2 * a + 1], pos, electric);
  return ci >= 0 ? 2 * a + 1 : -1;
}

// Column band state shared by the band loads and stores: y and z faces of the
// column (-1 if none), the band cells and their profile values b, a.
template <typename T>
struct ColBands {
  int yf, yci, zf, zci;
  T yb, ya, zb, za;
};

// Band state of column (j, k) for the H (ELECTRIC = false) or E update.
template <typename T, bool ELECTRIC>
__device__ __forceinline__ ColBands<T> col_bands(const Face<T>* face, int j, int k) {
  ColBands<T> cb;
  cb.yf = band_face(face, 1, j, ELECTRIC, cb.yci);
  cb.zf = band_face(face, 2, k, ELECTRIC, cb.zci);
  band_profile<T, ELECTRIC>(face, cb.yf, cb.yci, cb.yb, cb.ya);
  band_profile<T, ELECTRIC>(face, cb.zf, cb.zci, cb.zb, cb.za);
  return cb;
}

// Source boxes that contain this thread's (j, k) for component `comp` (bit mask).
template <typename T>
__device__ __forceinline__ unsigned source_columns(const Sources<T>& s, int comp, int j, int k) {
  unsigned m = 0;
  for (int q = 0; q < s.n; q++) {
    const SourceBox& b = s.box[q];
    if (b.comp == comp && j >= b.j0 && j <= b.j1 && k >= b.k0 && k <= b.k1) m |= 1u << q;
  }
  return m;
}

template <typename T>
__device__ __forceinline__ void inject_masked(const Sources<T>& s, unsigned mask, int i, int j, int k, int ts, T& e) {
  for (int q = 0; q < s.n; q++) {
    if (!(mask >> q & 1u)) continue;
    const SourceBox& b = s.box[q];
    if (i < b.i0 || i > b.i1) continue;
    const int ni = b.i1 - b.i0 + 1, nj = b.j1 - b.j0 + 1;
    const int n = ((k - b.k0) * nj + (j - b.j0)) * ni + (i - b.i0);
    e = add(e, mul(s.cs[q][n], s.wave[q][ts]));
  }
}

// ---------------------------------------------------------------------------
// H half-step
// ---------------------------------------------------------------------------
// What a thread knows about its (j, k) column.
template <typename T>
struct HCol {
  int j, k, oa, ob;                // column offsets: j*nz+k (Hx Hy Ez), j*(nz+1)+k (Hz Ey Ex)
  bool hx_ok, hy_ok, hz_ok;        // which H components have this column
  int yn, yp, zn, zp;              // H-band cell of the y/z faces, or -1
  float kmy, kmz;                  // 1/kappa_m along y and z (table problems)
};

// H update of plane i of a column.  LEAN: no CPML band touches this plane of
// the warp's columns, so the band tests and corrections are compiled out (and
// every 1/kappa factor is exactly 1, so LEAN and full agree bit for bit).
template <typename T, class C, bool EXACT, bool LEAN>
__device__ __forceinline__ void h_plane(const StepParams<T, C>& p, const HCol<T>& c, int i, T& ez_c, T& ey_c) {
  using A = Ar<T, EXACT>;
  const int nx = p.g.nx, ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1, sEx = nyp1 * nzp1;
  const Fields<T>& f = p.f;
  const bool inx = i < nx;
  const T ez_n = (inx && c.hy_ok) ? f.Ez[(i + 1) * sHyEz + c.oa] : T(0);
  const T ey_n = (inx && c.hz_ok) ? f.Ey[(i + 1) * sHzEy + c.ob] : T(0);
  const int xn = LEAN ? -1 : band_ci(p.face[0], i, false), xp = LEAN ? -1 : band_ci(p.face[1], i, false);
  const float kmx = LEAN ? 1.f : p.coef.invk(3, i);
  const T dx = p.dcell[0], dy = p.dcell[1], dz = p.dcell[2];
  T c0, c1, c2, u1, u2;
  // Hx (nx+1, ny, nz)
  if (c.hx_ok) {
    const int idx = i * sHx + c.oa;
    const T dey = A::dif(f.Ey[i * sHzEy + c.ob + 1], ey_c);
    const T dez = A::dif(f.Ez[i * sHyEz + c.oa + nz], ez_c);
    p.coef.get(0, idx, c.kmz, c.kmy, c0, c1, c2, u1, u2);
    T h = A::lin3(c0, f.Hx[idx], c1, dey, c2, dez);
    if (!LEAN) {
      // y faces: Psi_hxy (nx+1, nc, nz) by dEz/dy; z faces: Psi_hxz (nx+1, ny, nc) by dEy/dz
      if (c.yn >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[2], c.yn, (i * p.face[2].nc + c.yn) * nz + c.k, 0, dez, u2, dy, h);
      if (c.yp >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[3], c.yp, (i * p.face[3].nc + c.yp) * nz + c.k, 0, dez, u2, dy, h);
      if (c.zn >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[4], c.zn, (i * ny + c.j) * p.face[4].nc + c.zn, 0, dey, u1, dz, h);
      if (c.zp >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[5], c.zp, (i * ny + c.j) * p.face[5].nc + c.zp, 0, dey, u1, dz, h);
    }
    f.Hx[idx] = h;
  }
  if (inx) {
    const int ex = i * sEx + c.ob;
    const T ex_c = f.Ex[ex];
    // Hy (nx, ny+1, nz)
    if (c.hy_ok) {
      const int idx = i * sHyEz + c.oa;
      const T dez = A::dif(ez_n, ez_c);
      const T dex = A::dif(f.Ex[ex + 1], ex_c);
      p.coef.get(1, idx, kmx, c.kmz, c0, c1, c2, u1, u2);
      T h = A::lin3(c0, f.Hy[idx], c1, dez, c2, dex);
      if (!LEAN) {
        // x faces: Psi_hyx (nc, ny+1, nz) by dEz/dx; z faces: Psi_hyz (nx, ny+1, nc) by dEx/dz
        if (xn >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[0], xn, xn * sHyEz + c.oa, 0, dez, u1, dx, h);
        if (xp >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[1], xp, xp * sHyEz + c.oa, 0, dez, u1, dx, h);
        if (c.zn >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[4], c.zn, (i * nyp1 + c.j) * p.face[4].nc + c.zn, 1, dex, u2, dz, h);
        if (c.zp >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[5], c.zp, (i * nyp1 + c.j) * p.face[5].nc + c.zp, 1, dex, u2, dz, h);
      }
      f.Hy[idx] = h;
    }
    // Hz (nx, ny, nz+1)
    if (c.hz_ok) {
      const int idx = i * sHzEy + c.ob;
      const T dex = A::dif(f.Ex[ex + nzp1], ex_c);
      const T dey = A::dif(ey_n, ey_c);
      p.coef.get(2, idx, c.kmy, kmx, c0, c1, c2, u1, u2);
      T h = A::lin3(c0, f.Hz[idx], c1, dex, c2, dey);
      if (!LEAN) {
        // x faces: Psi_hzx (nc, ny, nz+1) by dEy/dx; y faces: Psi_hzy (nx, nc, nz+1) by dEx/dy
        if (xn >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[0], xn, xn * sHzEy + c.ob, 1, dey, u2, dx, h);
        if (xp >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[1], xp, xp * sHzEy + c.ob, 1, dey, u2, dx, h);
        if (c.yn >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[2], c.yn, (i * p.face[2].nc + c.yn) * nzp1 + c.k, 1, dex, u1, dy, h);
        if (c.yp >= 0) cpml_apply<T, C, EXACT, false>(p.coef, p.face[3], c.yp, (i * p.face[3].nc + c.yp) * nzp1 + c.k, 1, dex, u1, dy, h);
      }
      f.Hz[idx] = h;
    }
  }
  ez_c = ez_n;
  ey_c = ey_n;
}

// Inputs of one interior plane of an H column, loaded one plane ahead.
template <typename T, class C>
struct HIn {
  T hx, hy, hz, ey_kp, ez_jp, ex, ex_kp, ex_jp, ez_n, ey_n;
  typename C::Raw r0, r1, r2;
};

template <typename T, class C>
__device__ __forceinline__ void h_load(const StepParams<T, C>& p, const HCol<T>& c, int i, HIn<T, C>& in) {
  const int ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1, sEx = nyp1 * nzp1;
  const Fields<T>& f = p.f;
  const int ex = i * sEx + c.ob;
  in.ex = f.Ex[ex];
  if (c.hx_ok) {
    const int idx = i * sHx + c.oa;
    in.hx = f.Hx[idx];
    in.ey_kp = f.Ey[i * sHzEy + c.ob + 1];
    in.ez_jp = f.Ez[i * sHyEz + c.oa + nz];
    in.r0 = p.coef.fetch(0, idx);
  }
  if (c.hy_ok) {
    const int idx = i * sHyEz + c.oa;
    in.hy = f.Hy[idx];
    in.ex_kp = f.Ex[ex + 1];
    in.ez_n = f.Ez[idx + sHyEz];
    in.r1 = p.coef.fetch(1, idx);
  }
  if (c.hz_ok) {
    const int idx = i * sHzEy + c.ob;
    in.hz = f.Hz[idx];
    in.ex_jp = f.Ex[ex + nzp1];
    in.ey_n = f.Ey[idx + sHzEy];
    in.r2 = p.coef.fetch(2, idx);
  }
}

// Interior H plane (no CPML, kappa = 1): the same operations as h_plane<LEAN>.
template <typename T, class C, bool EXACT>
__device__ __forceinline__ void h_store(const StepParams<T, C>& p, const HCol<T>& c, int i, const HIn<T, C>& in,
                                        T& ez_c, T& ey_c) {
  using A = Ar<T, EXACT>;
  const int ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1;
  const Fields<T>& f = p.f;
  T c0, c1, c2;
  if (c.hx_ok) {
    p.coef.decode(0, in.r0, c0, c1, c2);
    f.Hx[i * sHx + c.oa] = A::lin3(c0, in.hx, c1, A::dif(in.ey_kp, ey_c), c2, A::dif(in.ez_jp, ez_c));
  }
  if (c.hy_ok) {
    p.coef.decode(1, in.r1, c0, c1, c2);
    f.Hy[i * sHyEz + c.oa] = A::lin3(c0, in.hy, c1, A::dif(in.ez_n, ez_c), c2, A::dif(in.ex_kp, in.ex));
  }
  if (c.hz_ok) {
    p.coef.decode(2, in.r2, c0, c1, c2);
    f.Hz[i * sHzEy + c.ob] = A::lin3(c0, in.hz, c1, A::dif(in.ex_jp, in.ex), c2, A::dif(in.ey_n, ey_c));
  }
  ez_c = in.ez_n;
  ey_c = in.ey_n;
}

// Every input of one H plane of a column in the full form (CPML bands, kappa),
// so that all loads of a plane can be issued before any of its stores.
template <typename T, class C>
struct HBand {
  HIn<T, C> v;          // field values and coefficient raws
  float kmx;            // 1/kappa_m at plane i
  int xf, xci;          // x band of plane i: face and cell, or -1
  T xb, xa;             // its profile values
  T pa[3], pb[3];       // Psi of the first / second correcting face of Hx, Hy, Hz
  T ca[3], cb[3];       // their CPsi (per-cell layouts; unused with tables)
};

// Face mask F of a band plane: bit 0 = an x band may hold the plane (uniform
// over the warp), bit 1 = the warp's row lies in a y band, bit 2 = some lane
// of the warp lies in a z band.  Faces outside the mask are compiled out;
// faces inside it are still tested per lane.
constexpr unsigned kFX = 1, kFY = 2, kFZ = 4, kFAll = 7;

template <typename T, class C, unsigned F = kFAll>
__device__ __forceinline__ void h_band_load(const StepParams<T, C>& p, const HCol<T>& c, const ColBands<T>& cb, int i,
                                            HBand<T, C>& in) {
  const int nx = p.g.nx, ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1, sEx = nyp1 * nzp1;
  const Fields<T>& f = p.f;
  if (F & kFX) {
    in.xf = band_face(p.face, 0, i, false, in.xci);
    band_profile<T, false>(p.face, in.xf, in.xci, in.xb, in.xa);
    in.kmx = p.coef.invk(3, i);
  } else {
    in.xf = -1;
    in.xci = 0;
    in.kmx = 1.f;
  }
  in.v.ez_n = T(0);
  in.v.ey_n = T(0);
  if (c.hx_ok) {
    const int idx = i * sHx + c.oa;
    in.v.hx = f.Hx[idx];
    in.v.ey_kp = f.Ey[i * sHzEy + c.ob + 1];
    in.v.ez_jp = f.Ez[i * sHyEz + c.oa + nz];
    in.v.r0 = p.coef.fetch(0, idx);
    if ((F & kFY) && cb.yf >= 0) {
      const Face<T>& fc = p.face[cb.yf];
      const int pi = (i * fc.nc + cb.yci) * nz + c.k;
      in.pa[0] = fc.psi[0][pi];
      in.ca[0] = p.coef.cpsi_fetch(fc, 0, pi);
    }
    if ((F & kFZ) && cb.zf >= 0) {
      const Face<T>& fc = p.face[cb.zf];
      const int pi = (i * ny + c.j) * fc.nc + cb.zci;
      in.pb[0] = fc.psi[0][pi];
      in.cb[0] = p.coef.cpsi_fetch(fc, 0, pi);
    }
  }
  if (i < nx) {
    const int ex = i * sEx + c.ob;
    in.v.ex = f.Ex[ex];
    if (c.hy_ok) {
      const int idx = i * sHyEz + c.oa;
      in.v.hy = f.Hy[idx];
      in.v.ex_kp = f.Ex[ex + 1];
      in.v.ez_n = f.Ez[idx + sHyEz];
      in.v.r1 = p.coef.fetch(1, idx);
      if (in.xf >= 0) {
        const Face<T>& fc = p.face[in.xf];
        const int pi = in.xci * sHyEz + c.oa;
        in.pa[1] = fc.psi[0][pi];
        in.ca[1] = p.coef.cpsi_fetch(fc, 0, pi);
      }
      if ((F & kFZ) && cb.zf >= 0) {
        const Face<T>& fc = p.face[cb.zf];
        const int pi = (i * nyp1 + c.j) * fc.nc + cb.zci;
        in.pb[1] = fc.psi[1][pi];
        in.cb[1] = p.coef.cpsi_fetch(fc, 1, pi);
      }
    }
    if (c.hz_ok) {
      const int idx = i * sHzEy + c.ob;
      in.v.hz = f.Hz[idx];
      in.v.ex_jp = f.Ex[ex + nzp1];
      in.v.ey_n = f.Ey[idx + sHzEy];
      in.v.r2 = p.coef.fetch(2, idx);
      if (in.xf >= 0) {
        const Face<T>& fc = p.face[in.xf];
        const int pi = in.xci * sHzEy + c.ob;
        in.pa[2] = fc.psi[1][pi];
        in.ca[2] = p.coef.cpsi_fetch(fc, 1, pi);
      }
      if ((F & kFY) && cb.yf >= 0) {
        const Face<T>& fc = p.face[cb.yf];
        const int pi = (i * fc.nc + cb.yci) * nzp1 + c.k;
        in.pb[2] = fc.psi[1][pi];
        in.cb[2] = p.coef.cpsi_fetch(fc, 1, pi);
      }
    }
  }
}

// h_plane<LEAN=false> on preloaded inputs (bands disjoint): identical
// arithmetic in the identical order.
template <typename T, class C, bool EXACT, unsigned F = kFAll>
__device__ __forceinline__ void h_band_store(const StepParams<T, C>& p, const HCol<T>& c, const ColBands<T>& cb, int i,
                                             const HBand<T, C>& in, T& ez_c, T& ey_c) {
  const float kmy = (F & kFY) ? c.kmy : 1.f, kmz = (F & kFZ) ? c.kmz : 1.f;
  using A = Ar<T, EXACT>;
  const int nx = p.g.nx, ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1;
  const Fields<T>& f = p.f;
  const T dx = p.dcell[0], dy = p.dcell[1], dz = p.dcell[2];
  T c0, c1, c2, u1, u2;
  if (c.hx_ok) {
    const T dey = A::dif(in.v.ey_kp, ey_c);
    const T dez = A::dif(in.v.ez_jp, ez_c);
    p.coef.decode_k(0, in.v.r0, kmz, kmy, c0, c1, c2, u1, u2);
    T h = A::lin3(c0, in.v.hx, c1, dey, c2, dez);
    if ((F & kFY) && cb.yf >= 0) {
      const Face<T>& fc = p.face[cb.yf];
      cpml_fold<T, C, EXACT>(p.coef, fc.psi[0] + (i * fc.nc + cb.yci) * nz + c.k, cb.yb, cb.ya, in.pa[0], in.ca[0], dez,
                             u2, dy, h);
    }
    if ((F & kFZ) && cb.zf >= 0) {
      const Face<T>& fc = p.face[cb.zf];
      cpml_fold<T, C, EXACT>(p.coef, fc.psi[0] + (i * ny + c.j) * fc.nc + cb.zci, cb.zb, cb.za, in.pb[0], in.cb[0], dey,
                             u1, dz, h);
    }
    f.Hx[i * sHx + c.oa] = h;
  }
  if (i < nx) {
    if (c.hy_ok) {
      const T dez = A::dif(in.v.ez_n, ez_c);
      const T dex = A::dif(in.v.ex_kp, in.v.ex);
      p.coef.decode_k(1, in.v.r1, in.kmx, kmz, c0, c1, c2, u1, u2);
      T h = A::lin3(c0, in.v.hy, c1, dez, c2, dex);
      if ((F & kFX) && in.xf >= 0)
        cpml_fold<T, C, EXACT>(p.coef, p.face[in.xf].psi[0] + in.xci * sHyEz + c.oa, in.xb, in.xa, in.pa[1], in.ca[1],
                               dez, u1, dx, h);
      if ((F & kFZ) && cb.zf >= 0) {
        const Face<T>& fc = p.face[cb.zf];
        cpml_fold<T, C, EXACT>(p.coef, fc.psi[1] + (i * nyp1 + c.j) * fc.nc + cb.zci, cb.zb, cb.za, in.pb[1], in.cb[1],
                               dex, u2, dz, h);
      }
      f.Hy[i * sHyEz + c.oa] = h;
    }
    if (c.hz_ok) {
      const T dex = A::dif(in.v.ex_jp, in.v.ex);
      const T dey = A::dif(in.v.ey_n, ey_c);
      p.coef.decode_k(2, in.v.r2, kmy, in.kmx, c0, c1, c2, u1, u2);
      T h = A::lin3(c0, in.v.hz, c1, dex, c2, dey);
      if ((F & kFX) && in.xf >= 0)
        cpml_fold<T, C, EXACT>(p.coef, p.face[in.xf].psi[1] + in.xci * sHzEy + c.ob, in.xb, in.xa, in.pa[2], in.ca[2],
                               dey, u2, dx, h);
      if ((F & kFY) && cb.yf >= 0) {
        const Face<T>& fc = p.face[cb.yf];
        cpml_fold<T, C, EXACT>(p.coef, fc.psi[1] + (i * fc.nc + cb.yci) * nzp1 + c.k, cb.yb, cb.ya, in.pb[2], in.cb[2],
                               dex, u1, dy, h);
      }
      f.Hz[i * sHzEy + c.ob] = h;
    }
  }
  ez_c = in.v.ez_n;
  ey_c = in.v.ey_n;
}

// Planes [a, b) of a column in the band form: every load of a plane is
// issued before its stores; with BPF the next plane's loads are also in flight.
template <typename T, class C, bool EXACT, bool BPF, unsigned F = kFAll>
__device__ __forceinline__ void h_band_range(const StepParams<T, C>& p, const HCol<T>& c, const ColBands<T>& cb, int a,
                                             int b, T& ez_c, T& ey_c) {
  if (a >= b) return;
  HBand<T, C> cur, nxt;
  if (!BPF) {
    for (int i = a; i < b; i++) {
      h_band_load<T, C, F>(p, c, cb, i, cur);
      h_band_store<T, C, EXACT, F>(p, c, cb, i, cur, ez_c, ey_c);
    }
    return;
  }
  h_band_load<T, C, F>(p, c, cb, a, cur);
  for (int i = a; i < b; i++) {
    if (i + 1 < b) h_band_load<T, C, F>(p, c, cb, i + 1, nxt);
    h_band_store<T, C, EXACT, F>(p, c, cb, i, cur, ez_c, ey_c);
    cur = nxt;
  }
}

// The band form (all loads of a band plane issued before its stores) serves
// every coefficient layout whose CPML bands are disjoint per axis.
template <class C>
struct BandForm {
  static constexpr bool kUse = true;
  static constexpr bool kPrefetch = false;
};

// ---------------------------------------------------------------------------
// Interior planes staged through shared memory (material-table problems,
// prefetch depth S = 3 or 4): each thread copies its own column's inputs of
// the next S planes into private shared-memory slots with cp.async, so S
// planes of loads are in flight without holding registers.  A plane's words
// are then read back into an HIn / EIn and go through h_store / e_store, so
// the arithmetic is that of the register-prefetched form.
// ---------------------------------------------------------------------------
extern __shared__ float fdtd_stage_smem[];

__device__ __forceinline__ void cp4(float* dst, const void* src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// The 4-byte word holding id `idx` of a uint8 id array (the arrays are
// 4-byte aligned and padded by 4 bytes), and the id's byte in that word.
__device__ __forceinline__ const void* id_word(const unsigned char* ids, int idx) { return ids + (idx & ~3); }
__device__ __forceinline__ unsigned char id_of(float w, int idx) {
  return (unsigned char)(__float_as_uint(w) >> (8 * (idx & 3)));
}

constexpr int kStageWords = 13;  // words staged per plane of an H or E column

// Word v of a thread's plane slot lives at s[v * nthr]: consecutive threads
// use consecutive words, so the slots are free of bank conflicts.
__device__ __forceinline__ void h_stage(const StepParams<float, TableCoef>& p, const HCol<float>& c, int i, float* s,
                                        int nthr) {
  const int ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1, sEx = nyp1 * nzp1;
  const Fields<float>& f = p.f;
  const int ex = i * sEx + c.ob;
  cp4(s, f.Ex + ex);
  if (c.hx_ok) {
    const int idx = i * sHx + c.oa;
    cp4(s + 1 * nthr, f.Hx + idx);
    cp4(s + 2 * nthr, f.Ey + i * sHzEy + c.ob + 1);
    cp4(s + 3 * nthr, f.Ez + i * sHyEz + c.oa + nz);
    cp4(s + 4 * nthr, id_word(p.coef.ids[0], idx));
  }
  if (c.hy_ok) {
    const int idx = i * sHyEz + c.oa;
    cp4(s + 5 * nthr, f.Hy + idx);
    cp4(s + 6 * nthr, f.Ex + ex + 1);
    cp4(s + 7 * nthr, f.Ez + idx + sHyEz);
    cp4(s + 8 * nthr, id_word(p.coef.ids[1], idx));
  }
  if (c.hz_ok) {
    const int idx = i * sHzEy + c.ob;
    cp4(s + 9 * nthr, f.Hz + idx);
    cp4(s + 10 * nthr, f.Ex + ex + nzp1);
    cp4(s + 11 * nthr, f.Ey + idx + sHzEy);
    cp4(s + 12 * nthr, id_word(p.coef.ids[2], idx));
  }
}

__device__ __forceinline__ void h_unstage(const StepParams<float, TableCoef>& p, const HCol<float>& c, int i,
                                          const float* s, int nthr, HIn<float, TableCoef>& in) {
  const int ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  in.ex = s[0];
  if (c.hx_ok) {
    in.hx = s[1 * nthr];
    in.ey_kp = s[2 * nthr];
    in.ez_jp = s[3 * nthr];
    in.r0 = id_of(s[4 * nthr], i * ny * nz + c.oa);
  }
  if (c.hy_ok) {
    in.hy = s[5 * nthr];
    in.ex_kp = s[6 * nthr];
    in.ez_n = s[7 * nthr];
    in.r1 = id_of(s[8 * nthr], i * nyp1 * nz + c.oa);
  }
  if (c.hz_ok) {
    in.hz = s[9 * nthr];
    in.ex_jp = s[10 * nthr];
    in.ey_n = s[11 * nthr];
    in.r2 = id_of(s[12 * nthr], i * ny * nzp1 + c.ob);
  }
}

// Planes [xa, xb) of an H column with S planes of loads in flight.
template <int S>
__device__ __forceinline__ void h_staged_range(const StepParams<float, TableCoef>& p, const HCol<float>& c, int xa,
                                               int xb, float& ez_c, float& ey_c) {
  const int nthr = blockDim.x * blockDim.y;
  float* base = fdtd_stage_smem + threadIdx.y * blockDim.x + threadIdx.x;
  const int n = xb - xa;
  for (int q = 0; q < S; q++) {
    if (q < n) h_stage(p, c, xa + q, base + q * kStageWords * nthr, nthr);
    cp_commit();
  }
  for (int q = 0; q < n; q++) {
    float* slot = base + (q % S) * kStageWords * nthr;
    cp_wait<S - 1>();
    HIn<float, TableCoef> in;
    h_unstage(p, c, xa + q, slot, nthr, in);
    h_store<float, TableCoef, false>(p, c, xa + q, in, ez_c, ey_c);
    if (q + S < n) h_stage(p, c, xa + q + S, slot, nthr);
    cp_commit();
  }
}

// Bytes of dynamic shared memory the staged form needs for a block.
__host__ __device__ constexpr int stage_smem_bytes(int S, int threads) { return S * kStageWords * threads * 4; }

// ---------------------------------------------------------------------------
// Interior planes staged by bulk copies (material-table problems, prefetch
// mode 5, 32-wide blocks): each warp copies the rows its 32 columns read --
// Hx, Hy, Hz, Ey(j), Ex(j), Ex(j+1), Ez(j), Ez(j+1) and the three id rows of
// a plane -- into a ring of kBulkStages shared-memory slots with one
// cp.async.bulk per row (lanes issue them side by side), completing on an
// mbarrier per slot.  A row copy is widened to 16-byte boundaries (the bulk
// copy's alignment rule) and read back from the offset of its first element.
// The lanes then compute the plane from shared memory with the arithmetic of
// h_store.  Waits are bounded: a wait that runs out records a fault in the
// handle's status and the kernel carries on, so nothing hangs.
// ---------------------------------------------------------------------------
constexpr int kBulkStages = 4;
constexpr int kBulkRow = 40;     // floats per staged field row (a 33-value row widened to 16 B: at most 144 B)
constexpr int kBulkIdRow = 12;   // floats per staged id row (32 ids widened: at most 48 B)
constexpr int kBulkRows = 8;
constexpr int kBulkSlot = kBulkRows * kBulkRow + 3 * kBulkIdRow;  // floats per warp and stage
constexpr int kBulkSpin = 1 << 20;                                // try_wait rounds before a wait gives up

__host__ __device__ constexpr int bulk_smem_bytes(int threads) {
  return (threads / 32) * kBulkStages * (kBulkSlot * 4 + 8);
}

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of a slot barrier; false when it ran out.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  for (int it = 0; it < kBulkSpin; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// Orders this thread's earlier shared-memory reads before later bulk (async
// proxy) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// One row copy: `n` elements of `esz` bytes from `src`, widened to 16-byte
// boundaries, into `dst` (16-byte aligned), completing on `bar`.  Returns the
// bytes copied.
__device__ __forceinline__ unsigned bulk_row(void* dst, const void* src, int n, int esz, unsigned long long* bar) {
  const unsigned long long a = (unsigned long long)src;
  const unsigned mis = (unsigned)(a & 15);
  const unsigned bytes = (mis + (unsigned)(n * esz) + 15u) & ~15u;
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(a - mis), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
  return bytes;
}
// Offset, in elements, of the first element of a row copied from `src`.
__device__ __forceinline__ int bulk_off(const void* src, int esz) {
  return (int)(((unsigned long long)src & 15) / (unsigned)esz);
}

// Source of staged row t of plane i for the warp whose columns start at k0 in
// row j (nullptr: the row does not exist there).  Rows 3 and 4 are read at
// k + 1 too, so they hold 33 values.
__device__ __forceinline__ const void* h_bulk_src(const StepParams<float, TableCoef>& p, int t, int i, int j, int k0) {
  const int ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1, sEx = nyp1 * nzp1;
  const Fields<float>& f = p.f;
  const bool jin = j < ny;
  switch (t) {
    case 0: return jin ? (const void*)(f.Hx + (i * sHx + j * nz + k0)) : nullptr;
    case 1: return f.Hy + (i * sHyEz + j * nz + k0);
    case 2: return jin ? (const void*)(f.Hz + (i * sHzEy + j * nzp1 + k0)) : nullptr;
    case 3: return jin ? (const void*)(f.Ey + (i * sHzEy + j * nzp1 + k0)) : nullptr;
    case 4: return f.Ex + (i * sEx + j * nzp1 + k0);
    case 5: return jin ? (const void*)(f.Ex + (i * sEx + (j + 1) * nzp1 + k0)) : nullptr;
    case 6: return f.Ez + (i * sHyEz + j * nz + k0);
    case 7: return jin ? (const void*)(f.Ez + (i * sHyEz + (j + 1) * nz + k0)) : nullptr;
    case 8: return jin ? (const void*)(p.coef.ids[0] + (i * sHx + j * nz + k0)) : nullptr;
    case 9: return p.coef.ids[1] + (i * sHyEz + j * nz + k0);
    default: return jin ? (const void*)(p.coef.ids[2] + (i * sHzEy + j * nzp1 + k0)) : nullptr;
  }
}

// Staged row t of a slot: field rows first, then the three id rows.
__device__ __forceinline__ float* bulk_row_dst(float* slot, int t) {
  return t < kBulkRows ? slot + t * kBulkRow : slot + kBulkRows * kBulkRow + (t - kBulkRows) * kBulkIdRow;
}

// Lean planes [xa, xb) of the H columns of one warp, staged by bulk copies
// (see above).  Every valid lane of the warp calls it together; on return
// ez_c, ey_c hold Ez and Ey of plane xb, as after h_lean_range.
__device__ __forceinline__ void h_bulk_range(const StepParams<float, TableCoef>& p, const HCol<float>& c, int xa,
                                             int xb, float& ez_c, float& ey_c) {
  if (xa >= xb) return;
  using A = Ar<float, false>;
  const int ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1;
  const Fields<float>& f = p.f;
  const int lane = threadIdx.x, w = threadIdx.y;
  const int k0 = c.k - lane, j = c.j;
  const unsigned mask = __activemask();
  const int nact = __popc(mask);
  const int nwarps = blockDim.y;
  float* wbase = fdtd_stage_smem + w * kBulkStages * kBulkSlot;
  unsigned long long* bars =
      reinterpret_cast<unsigned long long*>(fdtd_stage_smem + nwarps * kBulkStages * kBulkSlot) + w * kBulkStages;
  if (lane == 0) {
    for (int q = 0; q < kBulkStages; q++) mbar_init(bars + q, 1);
    mbar_fence_init();
  }
  __syncwarp(mask);
  // stage q holds plane xa + q; stage n = xb - xa (plane xb) only its Ey, Ez rows
  const int n = xb - xa;
  auto fill = [&](int q) {
    float* slot = wbase + (q % kBulkStages) * kBulkSlot;
    unsigned long long* bar = bars + q % kBulkStages;
    unsigned bytes = 0;
    for (int t = lane; t < kBulkRows + 3; t += nact) {
      if (q == n && t != 3 && t != 6) continue;
      const void* src = h_bulk_src(p, t, xa + q, j, k0);
      if (src) bytes += bulk_row(bulk_row_dst(slot, t), src, (t == 3 || t == 4) ? 33 : 32, t < kBulkRows ? 4 : 1, bar);
    }
    bytes = __reduce_add_sync(mask, bytes);
    if (lane == 0) mbar_arrive_tx(bar, bytes);
  };
  auto rowf = [&](int q, int t) -> const float* {
    return bulk_row_dst(wbase + (q % kBulkStages) * kBulkSlot, t) + bulk_off(h_bulk_src(p, t, xa + q, j, k0), 4);
  };
  auto rowb = [&](int q, int t) -> const unsigned char* {
    return reinterpret_cast<const unsigned char*>(bulk_row_dst(wbase + (q % kBulkStages) * kBulkSlot, t)) +
           bulk_off(h_bulk_src(p, t, xa + q, j, k0), 1);
  };
  for (int q = 0; q < kBulkStages && q <= n; q++) fill(q);
  bool ok = mbar_wait(bars, 0);
  for (int q = 0; q < n; q++) {
    const int i = xa + q;
    // after a wait has run out no other is tried, so a fault costs one bound
    if (ok) ok = mbar_wait(bars + (q + 1) % kBulkStages, ((q + 1) / kBulkStages) & 1);
    float c0, c1, c2;
    const float ey_i = c.hx_ok || c.hz_ok ? rowf(q, 3)[lane] : 0.f;
    const float ez_i = rowf(q, 6)[lane];
    if (c.hx_ok) {
      p.coef.decode(0, rowb(q, 8)[lane], c0, c1, c2);
      f.Hx[i * sHx + c.oa] = A::lin3(c0, rowf(q, 0)[lane], c1, A::dif(rowf(q, 3)[lane + 1], ey_i), c2,
                                     A::dif(rowf(q, 7)[lane], ez_i));
    }
    const float ex = rowf(q, 4)[lane];
    if (c.hy_ok) {
      p.coef.decode(1, rowb(q, 9)[lane], c0, c1, c2);
      f.Hy[i * sHyEz + c.oa] = A::lin3(c0, rowf(q, 1)[lane], c1, A::dif(rowf(q + 1, 6)[lane], ez_i), c2,
                                       A::dif(rowf(q, 4)[lane + 1], ex));
    }
    if (c.hz_ok) {
      p.coef.decode(2, rowb(q, 10)[lane], c0, c1, c2);
      f.Hz[i * sHzEy + c.ob] = A::lin3(c0, rowf(q, 2)[lane], c1, A::dif(rowf(q, 5)[lane], ex), c2,
                                       A::dif(rowf(q + 1, 3)[lane], ey_i));
    }
    __syncwarp(mask);
    fence_proxy_async();
    if (q + kBulkStages <= n) fill(q + kBulkStages);
  }
  // the carried x-neighbours for the planes after the range: Ez, Ey of plane xb
  ez_c = c.hy_ok ? rowf(n, 6)[lane] : 0.f;
  ey_c = c.hz_ok ? rowf(n, 3)[lane] : 0.f;
  __syncwarp(mask);
  if (lane == 0)   // every phase has completed: the barriers' memory may be initialised again
    for (int q = 0; q < kBulkStages; q++)
      asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_addr(bars + q)) : "memory");
  __syncwarp(mask);
  if (!ok) atomicExch(p.fault, 4);   // the handle's status code: a device wait ran out
}

// Minimum resident 256-thread blocks per SM the register budget is fitted to:
// FP64 values need twice the registers; a deeper register prefetch holds one
// more plane; the shared-memory stages (PF 3, 4) hold theirs outside registers.
template <typename T, int PF>
struct MinBlocks {
  static constexpr int value = sizeof(T) == 8 ? 2 : (PF == 2 ? 3 : 4);
};

// Lean planes [xa, xb) of an H column: register prefetch (PF 1, 2) or
// shared-memory stages (PF 3, 4, material tables).
template <typename T, class C, bool EXACT, int PF>
__device__ __forceinline__ void h_lean_range(const StepParams<T, C>& p, const HCol<T>& c, int xa, int xb, T& ez_c,
                                             T& ey_c) {
  if constexpr (PF == 5 && C::kTable) {
    h_bulk_range(p, c, xa, xb, ez_c, ey_c);
  } else if constexpr (PF >= 3 && PF <= 4 && C::kTable) {
    h_staged_range<PF>(p, c, xa, xb, ez_c, ey_c);
  } else if ((PF == 1 || PF == 5) && xa < xb) {
    // software pipeline, depth 1, as two alternating register sets: the next
    // plane's loads are in flight while plane i is computed and stored, and
    // no set is copied into the other
    HIn<T, C> a, b;
    h_load(p, c, xa, a);
    int i = xa;
    for (; i + 1 < xb; i += 2) {
      h_load(p, c, i + 1, b);
      h_store<T, C, EXACT>(p, c, i, a, ez_c, ey_c);
      if (i + 2 < xb) h_load(p, c, i + 2, a);
      h_store<T, C, EXACT>(p, c, i + 1, b, ez_c, ey_c);
    }
    if (i < xb) h_store<T, C, EXACT>(p, c, i, a, ez_c, ey_c);
  } else if (xa < xb) {
    // software pipeline: the loads of the next PF planes are in flight while
    // plane i is computed and stored
    HIn<T, C> cur, nxt, nx2;
    h_load(p, c, xa, cur);
    if (PF == 2 && xa + 1 < xb) h_load(p, c, xa + 1, nxt);
    for (int i = xa; i < xb; i++) {
      if (PF == 1) {
        if (i + 1 < xb) h_load(p, c, i + 1, nxt);
      } else {
        if (i + 2 < xb) h_load(p, c, i + 2, nx2);
      }
      h_store<T, C, EXACT>(p, c, i, cur, ez_c, ey_c);
      cur = nxt;
      if (PF == 2) nxt = nx2;
    }
  }
}

// Planes [i0, i1) of an H column in the band form, for a warp whose y/z
// band membership is YZ: the edge planes (an x band may apply) with x added,
// the x-interior planes [xa, xb) with YZ only, or lean when YZ is empty.
template <typename T, class C, bool EXACT, int PF, unsigned YZ>
__device__ __forceinline__ void h_tile_planes(const StepParams<T, C>& p, const HCol<T>& c, const ColBands<T>& cb, int i0,
                                              int xa, int xb, int i1, T& ez_c, T& ey_c) {
  constexpr bool BPF = BandForm<C>::kPrefetch;
  h_band_range<T, C, EXACT, BPF, kFX | YZ>(p, c, cb, i0, xa, ez_c, ey_c);
  if constexpr (YZ == 0)
    h_lean_range<T, C, EXACT, PF>(p, c, xa, xb, ez_c, ey_c);
  else
    h_band_range<T, C, EXACT, BPF, YZ>(p, c, cb, xa, xb, ez_c, ey_c);
  h_band_range<T, C, EXACT, BPF, kFX | YZ>(p, c, cb, xb, i1, ez_c, ey_c);
}

// H update of one tile: columns (bx*width + tx, by*rows + ty), x planes from
// bz*ichunk.  PF: how many planes ahead the interior loop loads.
template <typename T, class C, bool EXACT, int PF>
__device__ __forceinline__ void step_h_tile(const StepParams<T, C>& p, int bx, int by, int bz) {
  const int k = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int i0 = bz * p.ichunk;
  const int nx = p.g.nx, ny = p.g.ny, nz = p.g.nz;
  const bool valid = j <= ny && k <= nz;
  HCol<T> c;
  c.j = j;
  c.k = k;
  c.oa = j * nz + k;
  c.ob = j * (nz + 1) + k;
  c.hx_ok = j < ny && k < nz;
  c.hy_ok = k < nz;
  c.hz_ok = j < ny;
  c.yn = band_ci(p.face[2], j, false);
  c.yp = band_ci(p.face[3], j, false);
  c.zn = band_ci(p.face[4], k, false);
  c.zp = band_ci(p.face[5], k, false);
  // a warp is 32 consecutive k of one j (or, in 16-wide blocks, 16 k of two
  // rows); band membership is tested per lane, the votes only pick the form
  const bool ycol = c.yn >= 0 || c.yp >= 0, zcol = c.zn >= 0 || c.zp >= 0;
  const bool warp_lean = __all_sync(0xffffffffu, !valid || (!ycol && !zcol));
  const bool warp_y = __any_sync(0xffffffffu, valid && ycol);
  const bool warp_z = __any_sync(0xffffffffu, valid && zcol);
  if (!valid) return;
  c.kmy = p.coef.invk(4, j);
  c.kmz = p.coef.invk(5, k);
  const int i1 = min(i0 + p.ichunk, nx + 1);
  // carried x-neighbours: Ez(i,j,k), Ey(i,j,k)
  T ez_c = c.hy_ok ? p.f.Ez[i0 * (ny + 1) * nz + c.oa] : T(0);
  T ey_c = c.hz_ok ? p.f.Ey[i0 * ny * (nz + 1) + c.ob] : T(0);
  // x-interior planes [xa, xb): outside both x bands and below nx
  const int lo = p.face[0].nc > 0 ? p.face[0].m_start + p.face[0].nc : 0;
  const int hi = p.face[1].nc > 0 ? p.face[1].m_start : nx;
  const int xa = min(max(i0, lo), i1);
  const int xb = max(xa, min(i1, hi));
  if (BandForm<C>::kUse && p.bands_disjoint != 0) {
    const ColBands<T> cb = col_bands<T, false>(p.face, j, k);
    if (warp_y) {
      if (warp_z)
        h_tile_planes<T, C, EXACT, PF, kFY | kFZ>(p, c, cb, i0, xa, xb, i1, ez_c, ey_c);
      else
        h_tile_planes<T, C, EXACT, PF, kFY>(p, c, cb, i0, xa, xb, i1, ez_c, ey_c);
    } else {
      if (warp_z)
        h_tile_planes<T, C, EXACT, PF, kFZ>(p, c, cb, i0, xa, xb, i1, ez_c, ey_c);
      else
        h_tile_planes<T, C, EXACT, PF, 0>(p, c, cb, i0, xa, xb, i1, ez_c, ey_c);
    }
    return;
  }
  // plane-at-a-time form for the band planes; lean interior for lean warps
  const int la = warp_lean ? xa : i1, lb = warp_lean ? xb : i1;
  for (int i = i0; i < la; i++) h_plane<T, C, EXACT, false>(p, c, i, ez_c, ey_c);
  h_lean_range<T, C, EXACT, PF>(p, c, la, lb, ez_c, ey_c);
  for (int i = lb; i < i1; i++) h_plane<T, C, EXACT, false>(p, c, i, ez_c, ey_c);
}

template <typename T, class C, bool EXACT, int PF>
__global__ void __launch_bounds__(256, MinBlocks<T, PF>::value) k_step_h(StepParams<T, C> p) {
  if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
    const int ts = *p.ts + 1;  // first kernel of a step advances the device step counter
    *p.ts = ts;
    // a block boundary: the previous block was flushed at the end of step ts - 1
    if (p.dft_block > 0 && ts % p.dft_block == 0) *p.dft_done = ts;
  }
  step_h_tile<T, C, EXACT, PF>(p, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// Mid-step: the bulk-updated Ex(i=0) plane and the port currents.
// ---------------------------------------------------------------------------
template <typename T, class C, bool EXACT>
__device__ __forceinline__ void step_mid_thread(const StepParams<T, C>& p, const Probes& probes, long long t) {
  using A = Ar<T, EXACT>;
  const int ts = *p.ts;
  const int ny = p.g.ny, nz = p.g.nz, nzp1 = nz + 1;
  const long long plane = (long long)ny * nzp1;
  if (t < plane) {
    const int j = (int)(t / nzp1), k = (int)(t % nzp1);
    const int idx = j * nzp1 + k;  // Ex(0, j, k)
    T e = p.f.Ex[idx];
    if (j >= 1 && k >= 1 && k < nz) {
      const T dhz = A::dif(p.f.Hz[j * nzp1 + k], p.f.Hz[(j - 1) * nzp1 + k]);
      const T dhy = A::dif(p.f.Hy[j * nz + k], p.f.Hy[j * nz + k - 1]);
      T c0, c1, c2, u1, u2;
      p.coef.get(3, idx, p.coef.invk(1, j), p.coef.invk(2, k), c0, c1, c2, u1, u2);
      e = A::lin3(c0, e, c1, dhz, c2, dhy);
    }
    p.ex0b[idx] = e;
  } else if (t - plane < probes.n_i) {
    current_probe(p.f, probes, (int)(t - plane), ts);
  }
}

template <typename T, class C, bool EXACT>
__global__ void __launch_bounds__(256) k_step_mid(StepParams<T, C> p, Probes probes) {
  step_mid_thread<T, C, EXACT>(p, probes, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------
// E half-step
// ---------------------------------------------------------------------------
template <typename T>
struct ECol {
  int j, k, oa, ob;
  bool jy, kz, ey_ok, ez_ok;       // interior in y / z, Ey / Ez exist in this column
  int yn, yp, zn, zp;              // E-band cell of the y/z faces, or -1
  float key, kez;                  // 1/kappa_e along y and z (table problems)
  unsigned sx, sy, sz;             // sources covering this column (Ex, Ey, Ez)
};

template <typename T, class C, bool EXACT, bool LEAN>
__device__ __forceinline__ void e_plane(const StepParams<T, C>& p, const ECol<T>& c, int i, int ts, T& hz_p, T& hy_p) {
  using A = Ar<T, EXACT>;
  const int nx = p.g.nx, ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1, sEx = nyp1 * nzp1;
  const Fields<T>& f = p.f;
  const bool inx = i < nx;
  const bool wall = !inx && p.x_wall;  // Ey, Ez at i = nx held at zero
  // Hz(i,j,k) and Hy(i,j,k); at i = nx the reference reads Ex(0,j,k) after its
  // bulk update and the start of the Hz array instead (one plane past Hz / Hy)
  T hz_i = T(0), hy_i = T(0);
  if (c.ey_ok) hz_i = inx ? f.Hz[i * sHzEy + c.ob] : p.ex0b[c.ob];
  if (c.ez_ok) hy_i = inx ? f.Hy[i * sHyEz + c.oa] : f.Hz[c.oa];
  const int xn = LEAN ? -1 : band_ci(p.face[0], i, true), xp = LEAN ? -1 : band_ci(p.face[1], i, true);
  const float kex = LEAN ? 1.f : p.coef.invk(0, i);
  const T hx_c = (c.ey_ok && c.ez_ok) ? f.Hx[i * sHx + c.oa] : T(0);
  const T dx = p.dcell[0], dy = p.dcell[1], dz = p.dcell[2];
  T c0, c1, c2, u1, u2;
  // Ex (nx, ny+1, nz+1): bulk on j in [1,ny), k in [1,nz)
  if (inx) {
    const int idx = i * sEx + c.ob;
    T e = f.Ex[idx];
    T dhz = T(0), dhy = T(0);
    if (c.jy) dhz = A::dif(hz_i, f.Hz[i * sHzEy + c.ob - nzp1]);
    if (c.kz) dhy = A::dif(hy_i, f.Hy[i * sHyEz + c.oa - 1]);
    p.coef.get(3, idx, c.key, c.kez, c0, c1, c2, u1, u2);
    if (c.jy && c.kz) e = A::lin3(c0, e, c1, dhz, c2, dhy);
    if (!LEAN) {
      // y faces: Psi_exy (nx, nc, nz+1) by dHz/dy; z faces: Psi_exz (nx, ny+1, nc) by dHy/dz
      if (c.yn >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[2], c.yn, (i * p.face[2].nc + c.yn) * nzp1 + c.k, 3, dhz, u1, dy, e);
      if (c.yp >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[3], c.yp, (i * p.face[3].nc + c.yp) * nzp1 + c.k, 3, dhz, u1, dy, e);
      if (c.zn >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[4], c.zn, (i * nyp1 + c.j) * p.face[4].nc + c.zn, 2, dhy, u2, dz, e);
      if (c.zp >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[5], c.zp, (i * nyp1 + c.j) * p.face[5].nc + c.zp, 2, dhy, u2, dz, e);
      if (c.sx) inject_masked(p.src, c.sx, i, c.j, c.k, ts, e);
    }
    f.Ex[idx] = e;
  }
  // Ey (nx+1, ny, nz+1): bulk on i in [1,nx], k in [1,nz)
  if (c.ey_ok && !wall) {
    const int idx = i * sHzEy + c.ob;
    T e = f.Ey[idx];
    T dhx = T(0), dhz = T(0);
    if (c.kz) dhx = A::dif(hx_c, f.Hx[i * sHx + c.oa - 1]);
    if (i >= 1) dhz = A::dif(hz_i, hz_p);
    p.coef.get(4, idx, c.kez, kex, c0, c1, c2, u1, u2);
    if (i >= 1 && c.kz) e = A::lin3(c0, e, c1, dhx, c2, dhz);
    if (!LEAN) {
      // x faces: Psi_eyx (nc, ny, nz+1) by dHz/dx; z faces: Psi_eyz (nx+1, ny, nc) by dHx/dz
      if (xn >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[0], xn, xn * sHzEy + c.ob, 2, dhz, u2, dx, e);
      if (xp >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[1], xp, xp * sHzEy + c.ob, 2, dhz, u2, dx, e);
      if (c.zn >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[4], c.zn, (i * ny + c.j) * p.face[4].nc + c.zn, 3, dhx, u1, dz, e);
      if (c.zp >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[5], c.zp, (i * ny + c.j) * p.face[5].nc + c.zp, 3, dhx, u1, dz, e);
      if (c.sy) inject_masked(p.src, c.sy, i, c.j, c.k, ts, e);
    }
    f.Ey[idx] = e;
  }
  // Ez (nx+1, ny+1, nz): bulk on i in [1,nx], j in [1,ny)
  if (c.ez_ok && !wall) {
    const int idx = i * sHyEz + c.oa;
    T e = f.Ez[idx];
    T dhy = T(0), dhx = T(0);
    if (i >= 1) dhy = A::dif(hy_i, hy_p);
    if (c.jy) dhx = A::dif(hx_c, f.Hx[i * sHx + c.oa - nz]);
    p.coef.get(5, idx, kex, c.key, c0, c1, c2, u1, u2);
    if (i >= 1 && c.jy) e = A::lin3(c0, e, c1, dhy, c2, dhx);
    if (!LEAN) {
      // x faces: Psi_ezx (nc, ny+1, nz) by dHy/dx; y faces: Psi_ezy (nx+1, nc, nz) by dHx/dy
      if (xn >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[0], xn, xn * sHyEz + c.oa, 3, dhy, u1, dx, e);
      if (xp >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[1], xp, xp * sHyEz + c.oa, 3, dhy, u1, dx, e);
      if (c.yn >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[2], c.yn, (i * p.face[2].nc + c.yn) * nz + c.k, 2, dhx, u2, dy, e);
      if (c.yp >= 0) cpml_apply<T, C, EXACT, true>(p.coef, p.face[3], c.yp, (i * p.face[3].nc + c.yp) * nz + c.k, 2, dhx, u2, dy, e);
      if (c.sz) inject_masked(p.src, c.sz, i, c.j, c.k, ts, e);
    }
    f.Ez[idx] = e;
  }
  hz_p = hz_i;
  hy_p = hy_i;
}

// Inputs of one interior plane (1 <= i < nx) of an E column, loaded one plane ahead.
template <typename T, class C>
struct EIn {
  T ex, ey, ez, hz, hy, hz_jm, hy_km, hx, hx_km, hx_jm;
  typename C::Raw r0, r1, r2;
};

template <typename T, class C>
__device__ __forceinline__ void e_load(const StepParams<T, C>& p, const ECol<T>& c, int i, EIn<T, C>& in) {
  const int ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1, sEx = nyp1 * nzp1;
  const Fields<T>& f = p.f;
  if (c.jy && c.kz) {
    const int idx = i * sEx + c.ob;
    in.ex = f.Ex[idx];
    in.r0 = p.coef.fetch(3, idx);
  }
  if (c.ey_ok) in.hz = f.Hz[i * sHzEy + c.ob];
  if (c.ez_ok) in.hy = f.Hy[i * sHyEz + c.oa];
  if (c.jy) in.hz_jm = f.Hz[i * sHzEy + c.ob - nzp1];
  if (c.kz) in.hy_km = f.Hy[i * sHyEz + c.oa - 1];
  if (c.ey_ok && c.ez_ok) in.hx = f.Hx[i * sHx + c.oa];
  if (c.kz && c.ey_ok) {
    const int idx = i * sHzEy + c.ob;
    in.ey = f.Ey[idx];
    in.hx_km = f.Hx[i * sHx + c.oa - 1];
    in.r1 = p.coef.fetch(4, idx);
  }
  if (c.jy && c.ez_ok) {
    const int idx = i * sHyEz + c.oa;
    in.ez = f.Ez[idx];
    in.hx_jm = f.Hx[i * sHx + c.oa - nz];
    in.r2 = p.coef.fetch(5, idx);
  }
}

__device__ __forceinline__ void e_stage(const StepParams<float, TableCoef>& p, const ECol<float>& c, int i, float* s,
                                        int nthr) {
  const int ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1, sEx = nyp1 * nzp1;
  const Fields<float>& f = p.f;
  if (c.jy && c.kz) {
    const int idx = i * sEx + c.ob;
    cp4(s, f.Ex + idx);
    cp4(s + 1 * nthr, id_word(p.coef.ids[3], idx));
  }
  if (c.ey_ok) cp4(s + 2 * nthr, f.Hz + i * sHzEy + c.ob);
  if (c.ez_ok) cp4(s + 3 * nthr, f.Hy + i * sHyEz + c.oa);
  if (c.jy) cp4(s + 4 * nthr, f.Hz + i * sHzEy + c.ob - nzp1);
  if (c.kz) cp4(s + 5 * nthr, f.Hy + i * sHyEz + c.oa - 1);
  if (c.ey_ok && c.ez_ok) cp4(s + 6 * nthr, f.Hx + i * sHx + c.oa);
  if (c.kz && c.ey_ok) {
    const int idx = i * sHzEy + c.ob;
    cp4(s + 7 * nthr, f.Ey + idx);
    cp4(s + 8 * nthr, f.Hx + i * sHx + c.oa - 1);
    cp4(s + 9 * nthr, id_word(p.coef.ids[4], idx));
  }
  if (c.jy && c.ez_ok) {
    const int idx = i * sHyEz + c.oa;
    cp4(s + 10 * nthr, f.Ez + idx);
    cp4(s + 11 * nthr, f.Hx + i * sHx + c.oa - nz);
    cp4(s + 12 * nthr, id_word(p.coef.ids[5], idx));
  }
}

__device__ __forceinline__ void e_unstage(const StepParams<float, TableCoef>& p, const ECol<float>& c, int i,
                                          const float* s, int nthr, EIn<float, TableCoef>& in) {
  const int ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  if (c.jy && c.kz) {
    in.ex = s[0];
    in.r0 = id_of(s[1 * nthr], i * nyp1 * nzp1 + c.ob);
  }
  if (c.ey_ok) in.hz = s[2 * nthr];
  if (c.ez_ok) in.hy = s[3 * nthr];
  if (c.jy) in.hz_jm = s[4 * nthr];
  if (c.kz) in.hy_km = s[5 * nthr];
  if (c.ey_ok && c.ez_ok) in.hx = s[6 * nthr];
  if (c.kz && c.ey_ok) {
    in.ey = s[7 * nthr];
    in.hx_km = s[8 * nthr];
    in.r1 = id_of(s[9 * nthr], i * ny * nzp1 + c.ob);
  }
  if (c.jy && c.ez_ok) {
    in.ez = s[10 * nthr];
    in.hx_jm = s[11 * nthr];
    in.r2 = id_of(s[12 * nthr], i * nyp1 * nz + c.oa);
  }
}

// Interior E plane (no CPML, no source, 1 <= i < nx): the same operations as
// e_plane<LEAN>; values that the bulk update leaves alone are not rewritten.
template <typename T, class C, bool EXACT>
__device__ __forceinline__ void e_store(const StepParams<T, C>& p, const ECol<T>& c, int i, const EIn<T, C>& in,
                                        T& hz_p, T& hy_p) {
  using A = Ar<T, EXACT>;
  const int ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHyEz = nyp1 * nz, sHzEy = ny * nzp1, sEx = nyp1 * nzp1;
  const Fields<T>& f = p.f;
  T c0, c1, c2;
  if (c.jy && c.kz) {
    p.coef.decode(3, in.r0, c0, c1, c2);
    f.Ex[i * sEx + c.ob] = A::lin3(c0, in.ex, c1, A::dif(in.hz, in.hz_jm), c2, A::dif(in.hy, in.hy_km));
  }
  if (c.kz && c.ey_ok) {
    p.coef.decode(4, in.r1, c0, c1, c2);
    f.Ey[i * sHzEy + c.ob] = A::lin3(c0, in.ey, c1, A::dif(in.hx, in.hx_km), c2, A::dif(in.hz, hz_p));
  }
  if (c.jy && c.ez_ok) {
    p.coef.decode(5, in.r2, c0, c1, c2);
    f.Ez[i * sHyEz + c.oa] = A::lin3(c0, in.ez, c1, A::dif(in.hy, hy_p), c2, A::dif(in.hx, in.hx_jm));
  }
  hz_p = in.hz;
  hy_p = in.hy;
}

// Every input of one E plane of a column in the full form.
template <typename T, class C>
struct EBand {
  T ex, hz_jm, hy_km;   // Ex(i), Hz(i,j-1), Hy(i,k-1)
  T hz_i, hy_i, hx_c;   // Hz(i), Hy(i) (the reference's reads at i = nx), Hx(i)
  T ey, hx_km;          // Ey(i), Hx(i,k-1)
  T ez, hx_jm;          // Ez(i), Hx(i,j-1)
  typename C::Raw r0, r1, r2;
  float kex;            // 1/kappa_e at plane i
  int xf, xci;          // x band of plane i, or -1
  T xb, xa;             // its profile values
  T pa[3], pb[3];       // Psi of the first / second correcting face of Ex, Ey, Ez
  T ca[3], cb[3];
};

template <typename T, class C, unsigned F = kFAll>
__device__ __forceinline__ void e_band_load(const StepParams<T, C>& p, const ECol<T>& c, const ColBands<T>& cb, int i,
                                            EBand<T, C>& in) {
  const int nx = p.g.nx, ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHx = ny * nz, sHyEz = nyp1 * nz, sHzEy = ny * nzp1, sEx = nyp1 * nzp1;
  const Fields<T>& f = p.f;
  const bool inx = i < nx;
  in.hz_i = c.ey_ok ? (inx ? f.Hz[i * sHzEy + c.ob] : p.ex0b[c.ob]) : T(0);
  in.hy_i = c.ez_ok ? (inx ? f.Hy[i * sHyEz + c.oa] : f.Hz[c.oa]) : T(0);
  if (F & kFX) {
    in.xf = band_face(p.face, 0, i, true, in.xci);
    band_profile<T, true>(p.face, in.xf, in.xci, in.xb, in.xa);
    in.kex = p.coef.invk(0, i);
  } else {
    in.xf = -1;
    in.xci = 0;
    in.kex = 1.f;
  }
  in.hx_c = (c.ey_ok && c.ez_ok) ? f.Hx[i * sHx + c.oa] : T(0);
  if (inx) {
    const int idx = i * sEx + c.ob;
    in.ex = f.Ex[idx];
    if (c.jy) in.hz_jm = f.Hz[i * sHzEy + c.ob - nzp1];
    if (c.kz) in.hy_km = f.Hy[i * sHyEz + c.oa - 1];
    in.r0 = p.coef.fetch(3, idx);
    if ((F & kFY) && cb.yf >= 0) {
      const Face<T>& fc = p.face[cb.yf];
      const int pi = (i * fc.nc + cb.yci) * nzp1 + c.k;
      in.pa[0] = fc.psi[3][pi];
      in.ca[0] = p.coef.cpsi_fetch(fc, 3, pi);
    }
    if ((F & kFZ) && cb.zf >= 0) {
      const Face<T>& fc = p.face[cb.zf];
      const int pi = (i * nyp1 + c.j) * fc.nc + cb.zci;
      in.pb[0] = fc.psi[2][pi];
      in.cb[0] = p.coef.cpsi_fetch(fc, 2, pi);
    }
  }
  if (c.ey_ok) {
    const int idx = i * sHzEy + c.ob;
    in.ey = f.Ey[idx];
    if (c.kz) in.hx_km = f.Hx[i * sHx + c.oa - 1];
    in.r1 = p.coef.fetch(4, idx);
    if ((F & kFX) && in.xf >= 0) {
      const Face<T>& fc = p.face[in.xf];
      const int pi = in.xci * sHzEy + c.ob;
      in.pa[1] = fc.psi[2][pi];
      in.ca[1] = p.coef.cpsi_fetch(fc, 2, pi);
    }
    if ((F & kFZ) && cb.zf >= 0) {
      const Face<T>& fc = p.face[cb.zf];
      const int pi = (i * ny + c.j) * fc.nc + cb.zci;
      in.pb[1] = fc.psi[3][pi];
      in.cb[1] = p.coef.cpsi_fetch(fc, 3, pi);
    }
  }
  if (c.ez_ok) {
    const int idx = i * sHyEz + c.oa;
    in.ez = f.Ez[idx];
    if (c.jy) in.hx_jm = f.Hx[i * sHx + c.oa - nz];
    in.r2 = p.coef.fetch(5, idx);
    if ((F & kFX) && in.xf >= 0) {
      const Face<T>& fc = p.face[in.xf];
      const int pi = in.xci * sHyEz + c.oa;
      in.pa[2] = fc.psi[3][pi];
      in.ca[2] = p.coef.cpsi_fetch(fc, 3, pi);
    }
    if ((F & kFY) && cb.yf >= 0) {
      const Face<T>& fc = p.face[cb.yf];
      const int pi = (i * fc.nc + cb.yci) * nz + c.k;
      in.pb[2] = fc.psi[2][pi];
      in.cb[2] = p.coef.cpsi_fetch(fc, 2, pi);
    }
  }
}

// e_plane<LEAN=false> on preloaded inputs (bands disjoint): identical
// arithmetic in the identical order.
template <typename T, class C, bool EXACT, unsigned F = kFAll>
__device__ __forceinline__ void e_band_store(const StepParams<T, C>& p, const ECol<T>& c, const ColBands<T>& cb, int i,
                                             int ts, const EBand<T, C>& in, T& hz_p, T& hy_p) {
  const float key = (F & kFY) ? c.key : 1.f, kez = (F & kFZ) ? c.kez : 1.f;
  using A = Ar<T, EXACT>;
  const int nx = p.g.nx, ny = p.g.ny, nz = p.g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const int sHyEz = nyp1 * nz, sHzEy = ny * nzp1, sEx = nyp1 * nzp1;
  const Fields<T>& f = p.f;
  const T dx = p.dcell[0], dy = p.dcell[1], dz = p.dcell[2];
  T c0, c1, c2, u1, u2;
  if (i < nx) {
    T e = in.ex;
    const T dhz = c.jy ? A::dif(in.hz_i, in.hz_jm) : T(0);
    const T dhy = c.kz ? A::dif(in.hy_i, in.hy_km) : T(0);
    p.coef.decode_k(3, in.r0, key, kez, c0, c1, c2, u1, u2);
    if (c.jy && c.kz) e = A::lin3(c0, e, c1, dhz, c2, dhy);
    if ((F & kFY) && cb.yf >= 0) {
      const Face<T>& fc = p.face[cb.yf];
      cpml_fold<T, C, EXACT>(p.coef, fc.psi[3] + (i * fc.nc + cb.yci) * nzp1 + c.k, cb.yb, cb.ya, in.pa[0], in.ca[0],
                             dhz, u1, dy, e);
    }
    if ((F & kFZ) && cb.zf >= 0) {
      const Face<T>& fc = p.face[cb.zf];
      cpml_fold<T, C, EXACT>(p.coef, fc.psi[2] + (i * nyp1 + c.j) * fc.nc + cb.zci, cb.zb, cb.za, in.pb[0], in.cb[0],
                             dhy, u2, dz, e);
    }
    if (c.sx) inject_masked(p.src, c.sx, i, c.j, c.k, ts, e);
    f.Ex[i * sEx + c.ob] = e;
  }
  const bool wall = i >= nx && p.x_wall;  // Ey, Ez at i = nx held at zero
  if (c.ey_ok && !wall) {
    T e = in.ey;
    const T dhx = c.kz ? A::dif(in.hx_c, in.hx_km) : T(0);
    const T dhz = i >= 1 ? A::dif(in.hz_i, hz_p) : T(0);
    p.coef.decode_k(4, in.r1, kez, in.kex, c0, c1, c2, u1, u2);
    if (i >= 1 && c.kz) e = A::lin3(c0, e, c1, dhx, c2, dhz);
    if ((F & kFX) && in.xf >= 0)
      cpml_fold<T, C, EXACT>(p.coef, p.face[in.xf].psi[2] + in.xci * sHzEy + c.ob, in.xb, in.xa, in.pa[1], in.ca[1],
                             dhz, u2, dx, e);
    if ((F & kFZ) && cb.zf >= 0) {
      const Face<T>& fc = p.face[cb.zf];
      cpml_fold<T, C, EXACT>(p.coef, fc.psi[3] + (i * ny + c.j) * fc.nc + cb.zci, cb.zb, cb.za, in.pb[1], in.cb[1], dhx,
                             u1, dz, e);
    }
    if (c.sy) inject_masked(p.src, c.sy, i, c.j, c.k, ts, e);
    f.Ey[i * sHzEy + c.ob] = e;
  }
  if (c.ez_ok && !wall) {
    T e = in.ez;
    const T dhy = i >= 1 ? A::dif(in.hy_i, hy_p) : T(0);
    const T dhx = c.jy ? A::dif(in.hx_c, in.hx_jm) : T(0);
    p.coef.decode_k(5, in.r2, in.kex, key, c0, c1, c2, u1, u2);
    if (i >= 1 && c.jy) e = A::lin3(c0, e, c1, dhy, c2, dhx);
    if ((F & kFX) && in.xf >= 0)
      cpml_fold<T, C, EXACT>(p.coef, p.face[in.xf].psi[3] + in.xci * sHyEz + c.oa, in.xb, in.xa, in.pa[2], in.ca[2],
                             dhy, u1, dx, e);
    if ((F & kFY) && cb.yf >= 0) {
      const Face<T>& fc = p.face[cb.yf];
      cpml_fold<T, C, EXACT>(p.coef, fc.psi[2] + (i * fc.nc + cb.yci) * nz + c.k, cb.yb, cb.ya, in.pb[2], in.cb[2], dhx,
                             u2, dy, e);
    }
    if (c.sz) inject_masked(p.src, c.sz, i, c.j, c.k, ts, e);
    f.Ez[i * sHyEz + c.oa] = e;
  }
  hz_p = in.hz_i;
  hy_p = in.hy_i;
}

template <typename T, class C, bool EXACT, bool BPF, unsigned F = kFAll>
__device__ __forceinline__ void e_band_range(const StepParams<T, C>& p, const ECol<T>& c, const ColBands<T>& cb, int a,
                                             int b, int ts, T& hz_p, T& hy_p) {
  if (a >= b) return;
  EBand<T, C> cur, nxt;
  if (!BPF) {
    for (int i = a; i < b; i++) {
      e_band_load<T, C, F>(p, c, cb, i, cur);
      e_band_store<T, C, EXACT, F>(p, c, cb, i, ts, cur, hz_p, hy_p);
    }
    return;
  }
  e_band_load<T, C, F>(p, c, cb, a, cur);
  for (int i = a; i < b; i++) {
    if (i + 1 < b) e_band_load<T, C, F>(p, c, cb, i + 1, nxt);
    e_band_store<T, C, EXACT, F>(p, c, cb, i, ts, cur, hz_p, hy_p);
    cur = nxt;
  }
}

// Planes [xa, xb) of an E column with S planes of loads in flight.
template <int S>
__device__ __forceinline__ void e_staged_range(const StepParams<float, TableCoef>& p, const ECol<float>& c, int xa,
                                               int xb, float& hz_p, float& hy_p) {
  const int nthr = blockDim.x * blockDim.y;
  float* base = fdtd_stage_smem + threadIdx.y * blockDim.x + threadIdx.x;
  const int n = xb - xa;
  for (int q = 0; q < S; q++) {
    if (q < n) e_stage(p, c, xa + q, base + q * kStageWords * nthr, nthr);
    cp_commit();
  }
  for (int q = 0; q < n; q++) {
    float* slot = base + (q % S) * kStageWords * nthr;
    cp_wait<S - 1>();
    EIn<float, TableCoef> in;
    e_unstage(p, c, xa + q, slot, nthr, in);
    e_store<float, TableCoef, false>(p, c, xa + q, in, hz_p, hy_p);
    if (q + S < n) e_stage(p, c, xa + q + S, slot, nthr);
    cp_commit();
  }
}

// Lean planes [xa, xb) of an E column (1 <= i < nx, no band, no source).
template <typename T, class C, bool EXACT, int PF>
__device__ __forceinline__ void e_lean_range(const StepParams<T, C>& p, const ECol<T>& c, int xa, int xb, T& hz_p,
                                             T& hy_p) {
  if constexpr (PF >= 3 && PF <= 4 && C::kTable) {
    e_staged_range<PF>(p, c, xa, xb, hz_p, hy_p);
  } else if ((PF == 1 || PF == 5) && xa < xb) {
    // depth 1 as two alternating register sets (see h_lean_range)
    EIn<T, C> a, b;
    e_load(p, c, xa, a);
    int i = xa;
    for (; i + 1 < xb; i += 2) {
      e_load(p, c, i + 1, b);
      e_store<T, C, EXACT>(p, c, i, a, hz_p, hy_p);
      if (i + 2 < xb) e_load(p, c, i + 2, a);
      e_store<T, C, EXACT>(p, c, i + 1, b, hz_p, hy_p);
    }
    if (i < xb) e_store<T, C, EXACT>(p, c, i, a, hz_p, hy_p);
  } else if (xa < xb) {
    EIn<T, C> cur, nxt, nx2;
    e_load(p, c, xa, cur);
    if (PF == 2 && xa + 1 < xb) e_load(p, c, xa + 1, nxt);
    for (int i = xa; i < xb; i++) {
      if (PF == 1) {
        if (i + 1 < xb) e_load(p, c, i + 1, nxt);
      } else {
        if (i + 2 < xb) e_load(p, c, i + 2, nx2);
      }
      e_store<T, C, EXACT>(p, c, i, cur, hz_p, hy_p);
      cur = nxt;
      if (PF == 2) nxt = nx2;
    }
  }
}

// Planes [i0, i1) of an E column in the band form (see h_tile_planes); the
// edge ranges also hold the boundary planes i = 0 and i = nx.
template <typename T, class C, bool EXACT, int PF, unsigned YZ>
__device__ __forceinline__ void e_tile_planes(const StepParams<T, C>& p, const ECol<T>& c, const ColBands<T>& cb, int i0,
                                              int xa, int xb, int i1, int ts, T& hz_p, T& hy_p) {
  constexpr bool BPF = BandForm<C>::kPrefetch;
  e_band_range<T, C, EXACT, BPF, kFX | YZ>(p, c, cb, i0, xa, ts, hz_p, hy_p);
  if constexpr (YZ == 0)
    e_lean_range<T, C, EXACT, PF>(p, c, xa, xb, hz_p, hy_p);
  else
    e_band_range<T, C, EXACT, BPF, YZ>(p, c, cb, xa, xb, ts, hz_p, hy_p);
  e_band_range<T, C, EXACT, BPF, kFX | YZ>(p, c, cb, xb, i1, ts, hz_p, hy_p);
}

template <typename T, class C, bool EXACT, int PF>
__device__ __forceinline__ void step_e_tile(const StepParams<T, C>& p, int bx, int by, int bz) {
  const int k = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int i0 = bz * p.ichunk;
  const int nx = p.g.nx, ny = p.g.ny, nz = p.g.nz;
  const bool valid = j <= ny && k <= nz;
  ECol<T> c;
  c.j = j;
  c.k = k;
  c.oa = j * nz + k;
  c.ob = j * (nz + 1) + k;
  c.jy = j >= 1 && j < ny;
  c.kz = k >= 1 && k < nz;
  c.ey_ok = j < ny;
  c.ez_ok = k < nz;
  c.yn = band_ci(p.face[2], j, true);
  c.yp = band_ci(p.face[3], j, true);
  c.zn = band_ci(p.face[4], k, true);
  c.zp = band_ci(p.face[5], k, true);
  c.sx = source_columns(p.src, 0, j, k);
  c.sy = source_columns(p.src, 1, j, k);
  c.sz = source_columns(p.src, 2, j, k);
  const bool ycol = c.yn >= 0 || c.yp >= 0, zcol = c.zn >= 0 || c.zp >= 0, scol = (c.sx | c.sy | c.sz) != 0;
  const bool warp_lean = __all_sync(0xffffffffu, !valid || (!ycol && !zcol && !scol));
  const bool warp_y = __any_sync(0xffffffffu, valid && ycol);
  const bool warp_z = __any_sync(0xffffffffu, valid && zcol);
  const bool warp_src = __any_sync(0xffffffffu, valid && scol);
  if (!valid) return;
  c.key = p.coef.invk(1, j);
  c.kez = p.coef.invk(2, k);
  const int ts = *p.ts;
  const int i1 = min(i0 + p.ichunk, nx + 1);
  // carried x-neighbours: Hz(i-1,j,k), Hy(i-1,j,k)
  T hz_p = (i0 >= 1 && c.ey_ok) ? p.f.Hz[(i0 - 1) * ny * (nz + 1) + c.ob] : T(0);
  T hy_p = (i0 >= 1 && c.ez_ok) ? p.f.Hy[(i0 - 1) * (ny + 1) * nz + c.oa] : T(0);
  // x-interior planes [xa, xb): 1 <= i < nx and outside both x bands
  const int lo = p.face[0].nc > 0 ? p.face[0].e_start + p.face[0].nc : 1;
  const int hi = p.face[1].nc > 0 ? p.face[1].e_start : nx;
  const int xa = min(max(i0, max(lo, 1)), i1);
  const int xb = max(xa, min(i1, min(hi, nx)));
  if (BandForm<C>::kUse && p.bands_disjoint != 0) {
    const ColBands<T> cb = col_bands<T, true>(p.face, j, k);
    if (warp_src) {  // source columns: the general form on every plane
      e_band_range<T, C, EXACT, BandForm<C>::kPrefetch, kFAll>(p, c, cb, i0, i1, ts, hz_p, hy_p);
    } else if (warp_y) {
      if (warp_z)
        e_tile_planes<T, C, EXACT, PF, kFY | kFZ>(p, c, cb, i0, xa, xb, i1, ts, hz_p, hy_p);
      else
        e_tile_planes<T, C, EXACT, PF, kFY>(p, c, cb, i0, xa, xb, i1, ts, hz_p, hy_p);
    } else {
      if (warp_z)
        e_tile_planes<T, C, EXACT, PF, kFZ>(p, c, cb, i0, xa, xb, i1, ts, hz_p, hy_p);
      else
        e_tile_planes<T, C, EXACT, PF, 0>(p, c, cb, i0, xa, xb, i1, ts, hz_p, hy_p);
    }
    return;
  }
  // plane-at-a-time form for the band planes; lean interior for lean warps
  const int la = warp_lean ? xa : i1, lb = warp_lean ? xb : i1;
  for (int i = i0; i < la; i++) e_plane<T, C, EXACT, false>(p, c, i, ts, hz_p, hy_p);
  e_lean_range<T, C, EXACT, PF>(p, c, la, lb, hz_p, hy_p);
  for (int i = lb; i < i1; i++) e_plane<T, C, EXACT, false>(p, c, i, ts, hz_p, hy_p);
}

template <typename T, class C, bool EXACT, int PF>
__global__ void __launch_bounds__(256, MinBlocks<T, PF>::value) k_step_e(StepParams<T, C> p) {
  step_e_tile<T, C, EXACT, PF>(p, blockIdx.x, blockIdx.y, blockIdx.z);
}

}  // namespace fdtd
