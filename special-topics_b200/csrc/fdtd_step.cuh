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
// The kernels are generic over how a cell finds its update coefficients:
//   ArrayCoef<T>  the reference's 18 per-cell arrays (FP64 drop-in, FP32 legacy)
//   TableCoef     one uint8 material id per cell and component into a small
//                 coefficient table, with the CPML kappa division applied from
//                 1-D per-axis profiles (FP32 fast path)
// and over the arithmetic: EXACT uses the _rn intrinsics so that nvcc never
// fuses a multiply into an add and every cell sees the reference's sequence
// of rounded FP64 operations; otherwise FMA is allowed.
//
// Each thread owns one (i,j,k) of the (nx+1, ny+1, nz+1) box and updates the
// components that exist there, so every Psi element and field value has
// exactly one writer and the CPML corrections of a value are applied in the
// reference's face order xn xp yn yp zn zp.
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
// ---------------------------------------------------------------------------
template <typename T>
struct ArrayCoef {
  const T* c[6][3];  // [component][self, curl1, curl2]
  __device__ __forceinline__ void get(int comp, long long idx, int, int, T& c0, T& c1, T& c2, T& u1,
                                      T& u2) const {
    c0 = c[comp][0][idx];
    c1 = c[comp][1][idx];
    c2 = c[comp][2][idx];
    u1 = c1;
    u2 = c2;
  }
  // CPsi of Psi element pi of a face slot (the reference's per-element array)
  __device__ __forceinline__ T cpsi(const Face<T>& F, int slot, long long pi, T, T) const {
    return F.cpsi[slot][pi];
  }
};

constexpr int kTableRows = 256;

struct TableCoef {
  const unsigned char* ids[6];  // per component, field order
  const float* tab;             // [6][kTableRows][3] self, curl1, curl2 without kappa
  const float* invk[6];         // 1/kappa along x y z for E (0..2) and H (3..5), length n+1
  float d[3];                   // dx dy dz (CPsi = coefficient * cell size)
  // positions along the curl axes: pos1 / pos2 are passed by the kernel
  __device__ __forceinline__ void get(int comp, long long idx, int pos1, int pos2, float& c0, float& c1,
                                      float& c2, float& u1, float& u2) const {
    const int id = __ldg(ids[comp] + idx);
    const float* r = tab + (comp * kTableRows + id) * 3;
    c0 = __ldg(r);
    u1 = __ldg(r + 1);
    u2 = __ldg(r + 2);
    // axis of curl1 / curl2 per component (see table above)
    const int ax1 = comp == 0 ? 2 : comp == 1 ? 0 : comp == 2 ? 1 : comp == 3 ? 1 : comp == 4 ? 2 : 0;
    const int ax2 = comp == 0 ? 1 : comp == 1 ? 2 : comp == 2 ? 0 : comp == 3 ? 2 : comp == 4 ? 0 : 1;
    const int base = comp < 3 ? 3 : 0;
    c1 = u1 * __ldg(invk[base + ax1] + pos1);
    c2 = u2 * __ldg(invk[base + ax2] + pos2);
  }
  __device__ __forceinline__ float cpsi(const Face<float>& F, int, long long, float u, float dcell) const {
    return u * dcell;
  }
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
};

// CPML on one face for an H value: Psi update from `drive`, then H += CPsi*Psi.
template <typename T, class C, bool EXACT>
__device__ __forceinline__ void cpml_h(const C& coef, const Face<T>& F, int pos, long long pi_base,
                                       long long pi_stride_ci, int slot, T drive, T u, T dcell, T& h) {
  if (F.nc > 0 && pos >= F.m_start && pos < F.m_start + F.nc) {
    const int ci = pos - F.m_start;
    const long long pi = pi_base + (long long)ci * pi_stride_ci;
    T* P = F.psi[slot];
    const T ps = Ar<T, EXACT>::lin2(F.b_m[ci], P[pi], F.a_m[ci], drive);
    P[pi] = ps;
    h = Ar<T, EXACT>::axpy(h, coef.cpsi(F, slot, pi, u, dcell), ps);
  }
}

template <typename T, class C, bool EXACT>
__device__ __forceinline__ void cpml_e(const C& coef, const Face<T>& F, int pos, long long pi_base,
                                       long long pi_stride_ci, int slot, T drive, T u, T dcell, T& e) {
  if (F.nc > 0 && pos >= F.e_start && pos < F.e_start + F.nc) {
    const int ci = pos - F.e_start;
    const long long pi = pi_base + (long long)ci * pi_stride_ci;
    T* P = F.psi[slot];
    const T ps = Ar<T, EXACT>::lin2(F.b_e[ci], P[pi], F.a_e[ci], drive);
    P[pi] = ps;
    e = Ar<T, EXACT>::axpy(e, coef.cpsi(F, slot, pi, u, dcell), ps);
  }
}

template <typename T>
__device__ __forceinline__ bool in_e_band(const Face<T>& F, int pos) {
  return F.nc > 0 && pos >= F.e_start && pos < F.e_start + F.nc;
}

// ---------------------------------------------------------------------------
// H half-step
// ---------------------------------------------------------------------------
template <typename T, class C, bool EXACT>
__global__ void __launch_bounds__(256) k_step_h(StepParams<T, C> p) {
  using A = Ar<T, EXACT>;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z * blockDim.z + threadIdx.z;
  if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && threadIdx.y == 0 &&
      threadIdx.z == 0)
    *p.ts += 1;  // first kernel of a step advances the device step counter
  const GridDims& g = p.g;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const Fields<T>& f = p.f;
  T c0, c1, c2, u1, u2;

  // Hx (nx+1, ny, nz)
  if (j < ny && k < nz) {
    const long long idx = ((long long)i * ny + j) * nz + k;
    const long long ey = ((long long)i * ny + j) * nzp1 + k;
    const long long ez = ((long long)i * nyp1 + j) * nz + k;
    const T dey = A::dif(f.Ey[ey + 1], f.Ey[ey]);
    const T dez = A::dif(f.Ez[ez + nz], f.Ez[ez]);
    p.coef.get(0, idx, k, j, c0, c1, c2, u1, u2);
    T h = A::lin3(c0, f.Hx[idx], c1, dey, c2, dez);
    // y faces: Psi_hxy (nx+1, nc, nz) by dEz/dy; z faces: Psi_hxz (nx+1, ny, nc) by dEy/dz
    cpml_h<T, C, EXACT>(p.coef, p.face[2], j, (long long)i * p.face[2].nc * nz + k, nz, 0, dez, u2, p.dcell[1], h);
    cpml_h<T, C, EXACT>(p.coef, p.face[3], j, (long long)i * p.face[3].nc * nz + k, nz, 0, dez, u2, p.dcell[1], h);
    cpml_h<T, C, EXACT>(p.coef, p.face[4], k, ((long long)i * ny + j) * p.face[4].nc, 1, 0, dey, u1, p.dcell[2], h);
    cpml_h<T, C, EXACT>(p.coef, p.face[5], k, ((long long)i * ny + j) * p.face[5].nc, 1, 0, dey, u1, p.dcell[2], h);
    f.Hx[idx] = h;
  }
  // Hy (nx, ny+1, nz)
  if (i < nx && k < nz) {
    const long long idx = ((long long)i * nyp1 + j) * nz + k;
    const long long ex = ((long long)i * nyp1 + j) * nzp1 + k;
    const T dez = A::dif(f.Ez[idx + (long long)nyp1 * nz], f.Ez[idx]);  // Ez shares Hy's (j,k) layout
    const T dex = A::dif(f.Ex[ex + 1], f.Ex[ex]);
    p.coef.get(1, idx, i, k, c0, c1, c2, u1, u2);
    T h = A::lin3(c0, f.Hy[idx], c1, dez, c2, dex);
    // x faces: Psi_hyx (nc, ny+1, nz) by dEz/dx; z faces: Psi_hyz (nx, ny+1, nc) by dEx/dz
    cpml_h<T, C, EXACT>(p.coef, p.face[0], i, (long long)j * nz + k, (long long)nyp1 * nz, 0, dez, u1, p.dcell[0], h);
    cpml_h<T, C, EXACT>(p.coef, p.face[1], i, (long long)j * nz + k, (long long)nyp1 * nz, 0, dez, u1, p.dcell[0], h);
    cpml_h<T, C, EXACT>(p.coef, p.face[4], k, ((long long)i * nyp1 + j) * p.face[4].nc, 1, 1, dex, u2, p.dcell[2], h);
    cpml_h<T, C, EXACT>(p.coef, p.face[5], k, ((long long)i * nyp1 + j) * p.face[5].nc, 1, 1, dex, u2, p.dcell[2], h);
    f.Hy[idx] = h;
  }
  // Hz (nx, ny, nz+1)
  if (i < nx && j < ny) {
    const long long idx = ((long long)i * ny + j) * nzp1 + k;
    const long long ex = ((long long)i * nyp1 + j) * nzp1 + k;
    const T dex = A::dif(f.Ex[ex + nzp1], f.Ex[ex]);
    const T dey = A::dif(f.Ey[idx + (long long)ny * nzp1], f.Ey[idx]);  // Ey shares Hz's (j,k) layout
    p.coef.get(2, idx, j, i, c0, c1, c2, u1, u2);
    T h = A::lin3(c0, f.Hz[idx], c1, dex, c2, dey);
    // x faces: Psi_hzx (nc, ny, nz+1) by dEy/dx; y faces: Psi_hzy (nx, nc, nz+1) by dEx/dy
    cpml_h<T, C, EXACT>(p.coef, p.face[0], i, (long long)j * nzp1 + k, (long long)ny * nzp1, 1, dey, u2, p.dcell[0], h);
    cpml_h<T, C, EXACT>(p.coef, p.face[1], i, (long long)j * nzp1 + k, (long long)ny * nzp1, 1, dey, u2, p.dcell[0], h);
    cpml_h<T, C, EXACT>(p.coef, p.face[2], j, (long long)i * p.face[2].nc * nzp1 + k, nzp1, 1, dex, u1, p.dcell[1], h);
    cpml_h<T, C, EXACT>(p.coef, p.face[3], j, (long long)i * p.face[3].nc * nzp1 + k, nzp1, 1, dex, u1, p.dcell[1], h);
    f.Hz[idx] = h;
  }
}

// ---------------------------------------------------------------------------
// Mid-step: the bulk-updated Ex(i=0) plane and the port currents.
// ---------------------------------------------------------------------------
template <typename T, class C, bool EXACT>
__global__ void __launch_bounds__(256) k_step_mid(StepParams<T, C> p, Probes probes) {
  using A = Ar<T, EXACT>;
  const int ts = *p.ts;
  const GridDims& g = p.g;
  const int ny = g.ny, nz = g.nz, nzp1 = nz + 1;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long plane = (long long)ny * nzp1;
  if (t < plane) {
    const int j = (int)(t / nzp1), k = (int)(t % nzp1);
    const long long idx = (long long)j * nzp1 + k;  // Ex(0, j, k)
    T e = p.f.Ex[idx];
    if (j >= 1 && k >= 1 && k < nz) {
      const T dhz = A::dif(p.f.Hz[(long long)j * nzp1 + k], p.f.Hz[(long long)(j - 1) * nzp1 + k]);
      const T dhy = A::dif(p.f.Hy[(long long)j * nz + k], p.f.Hy[(long long)j * nz + k - 1]);
      T c0, c1, c2, u1, u2;
      p.coef.get(3, idx, j, k, c0, c1, c2, u1, u2);
      e = A::lin3(c0, e, c1, dhz, c2, dhy);
    }
    p.ex0b[idx] = e;
  } else if (t - plane < probes.n_i) {
    current_probe(p.f, probes, (int)(t - plane), ts);
  }
}

// ---------------------------------------------------------------------------
// E half-step
// ---------------------------------------------------------------------------
template <typename T, class C, bool EXACT>
__global__ void __launch_bounds__(256) k_step_e(StepParams<T, C> p) {
  using A = Ar<T, EXACT>;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z * blockDim.z + threadIdx.z;
  const GridDims& g = p.g;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  const int ts = *p.ts;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nyp1 = ny + 1, nzp1 = nz + 1;
  const Fields<T>& f = p.f;
  T c0, c1, c2, u1, u2;

  // Ex (nx, ny+1, nz+1): bulk on j in [1,ny), k in [1,nz); y-face and z-face CPML
  if (i < nx) {
    const long long idx = ((long long)i * nyp1 + j) * nzp1 + k;
    T e = f.Ex[idx];
    const bool jy = (j >= 1 && j < ny), kz = (k >= 1 && k < nz);
    T dhz = T(0), dhy = T(0);
    if (jy) dhz = A::dif(f.Hz[((long long)i * ny + j) * nzp1 + k], f.Hz[((long long)i * ny + j - 1) * nzp1 + k]);
    if (kz) dhy = A::dif(f.Hy[((long long)i * nyp1 + j) * nz + k], f.Hy[((long long)i * nyp1 + j) * nz + k - 1]);
    p.coef.get(3, idx, j, k, c0, c1, c2, u1, u2);
    if (jy && kz) e = A::lin3(c0, e, c1, dhz, c2, dhy);
    // y faces: Psi_exy (nx, nc, nz+1) by dHz/dy; z faces: Psi_exz (nx, ny+1, nc) by dHy/dz
    cpml_e<T, C, EXACT>(p.coef, p.face[2], j, (long long)i * p.face[2].nc * nzp1 + k, nzp1, 3, dhz, u1, p.dcell[1], e);
    cpml_e<T, C, EXACT>(p.coef, p.face[3], j, (long long)i * p.face[3].nc * nzp1 + k, nzp1, 3, dhz, u1, p.dcell[1], e);
    cpml_e<T, C, EXACT>(p.coef, p.face[4], k, ((long long)i * nyp1 + j) * p.face[4].nc, 1, 2, dhy, u2, p.dcell[2], e);
    cpml_e<T, C, EXACT>(p.coef, p.face[5], k, ((long long)i * nyp1 + j) * p.face[5].nc, 1, 2, dhy, u2, p.dcell[2], e);
    inject_sources(p.src, 0, i, j, k, ts, e);
    f.Ex[idx] = e;
  }
  // Ey (nx+1, ny, nz+1): bulk on i in [1,nx], k in [1,nz); x-face and z-face CPML
  if (j < ny) {
    const long long idx = ((long long)i * ny + j) * nzp1 + k;
    T e = f.Ey[idx];
    const bool kz = (k >= 1 && k < nz);
    const bool bulk = (i >= 1) && kz;
    const bool xb = in_e_band(p.face[0], i) || in_e_band(p.face[1], i);
    T dhx = T(0), dhz = T(0);
    if (kz) dhx = A::dif(f.Hx[((long long)i * ny + j) * nz + k], f.Hx[((long long)i * ny + j) * nz + k - 1]);
    if (bulk || xb) {
      // Hz(i=nx) does not exist; the reference reads Ex(0,j,k) there, after its bulk update
      const T hz1 = (i < nx) ? f.Hz[idx] : p.ex0b[(long long)j * nzp1 + k];  // Hz shares Ey's (j,k) layout
      dhz = A::dif(hz1, f.Hz[idx - (long long)ny * nzp1]);
    }
    p.coef.get(4, idx, k, i, c0, c1, c2, u1, u2);
    if (bulk) e = A::lin3(c0, e, c1, dhx, c2, dhz);
    // x faces: Psi_eyx (nc, ny, nz+1) by dHz/dx; z faces: Psi_eyz (nx+1, ny, nc) by dHx/dz
    cpml_e<T, C, EXACT>(p.coef, p.face[0], i, (long long)j * nzp1 + k, (long long)ny * nzp1, 2, dhz, u2, p.dcell[0], e);
    cpml_e<T, C, EXACT>(p.coef, p.face[1], i, (long long)j * nzp1 + k, (long long)ny * nzp1, 2, dhz, u2, p.dcell[0], e);
    cpml_e<T, C, EXACT>(p.coef, p.face[4], k, ((long long)i * ny + j) * p.face[4].nc, 1, 3, dhx, u1, p.dcell[2], e);
    cpml_e<T, C, EXACT>(p.coef, p.face[5], k, ((long long)i * ny + j) * p.face[5].nc, 1, 3, dhx, u1, p.dcell[2], e);
    inject_sources(p.src, 1, i, j, k, ts, e);
    f.Ey[idx] = e;
  }
  // Ez (nx+1, ny+1, nz): bulk on i in [1,nx], j in [1,ny); x-face and y-face CPML
  if (k < nz) {
    const long long idx = ((long long)i * nyp1 + j) * nz + k;
    T e = f.Ez[idx];
    const bool jy = (j >= 1 && j < ny);
    const bool bulk = (i >= 1) && jy;
    const bool xb = in_e_band(p.face[0], i) || in_e_band(p.face[1], i);
    T dhy = T(0), dhx = T(0);
    if (bulk || xb) {
      // Hy(i=nx) does not exist; the reference reads the Hz array from its start there
      const T hy1 = (i < nx) ? f.Hy[idx] : f.Hz[(long long)j * nz + k];  // Hy shares Ez's (j,k) layout
      dhy = A::dif(hy1, f.Hy[idx - (long long)nyp1 * nz]);
    }
    if (jy) dhx = A::dif(f.Hx[((long long)i * ny + j) * nz + k], f.Hx[((long long)i * ny + j - 1) * nz + k]);
    p.coef.get(5, idx, i, j, c0, c1, c2, u1, u2);
    if (bulk) e = A::lin3(c0, e, c1, dhy, c2, dhx);
    // x faces: Psi_ezx (nc, ny+1, nz) by dHy/dx; y faces: Psi_ezy (nx+1, nc, nz) by dHx/dy
    cpml_e<T, C, EXACT>(p.coef, p.face[0], i, (long long)j * nz + k, (long long)nyp1 * nz, 3, dhy, u1, p.dcell[0], e);
    cpml_e<T, C, EXACT>(p.coef, p.face[1], i, (long long)j * nz + k, (long long)nyp1 * nz, 3, dhy, u1, p.dcell[0], e);
    cpml_e<T, C, EXACT>(p.coef, p.face[2], j, (long long)i * p.face[2].nc * nz + k, nz, 2, dhx, u2, p.dcell[1], e);
    cpml_e<T, C, EXACT>(p.coef, p.face[3], j, (long long)i * p.face[3].nc * nz + k, nz, 2, dhx, u2, p.dcell[1], e);
    inject_sources(p.src, 2, i, j, k, ts, e);
    f.Ez[idx] = e;
  }
}

}  // namespace fdtd
