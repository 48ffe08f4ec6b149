// fdtd_material.cuh -- device side of the material-table construction.
//
// A cell's coefficient triple for a component is fixed by the materials of
// the cells its value averages (js_fdtd/src/materials.js:127-230):
//   Ex, Ey, Ez   4-cell arithmetic mean of eps_r and sigma_e on the interior
//                of the component array, fill values (1, 0) elsewhere
//   Hx, Hy, Hz   2-cell harmonic mean of mu_r and sigma_m on the interior,
//                fill values (1, 0) elsewhere
// and by the zero-thickness PEC plates that overwrite sigma_e on boxes of the
// E arrays (materials.js:253-332).  Pass 1 encodes each cell as an integer
// code (the ordered material tuple, or the fill code, times the plate that
// last covered it) and marks the codes that occur; the host turns the
// occurring codes into coefficient rows with the reference's formulas; pass 2
// writes each cell's row id.
#pragma once
#include <stdint.h>

namespace fdtd {

constexpr int kMaxPlates = 64;

struct PlateBox {
  int comp;  // 0=Ex 1=Ey 2=Ez
  int i0, i1, j0, j1, k0, k1;  // inclusive
  int sigma_id;                // index into the distinct plate conductivities (0-based)
};

struct MatBuild {
  const uint8_t* mat;  // material grid (nx, ny, nz), 1-based type ids
  int nx, ny, nz;
  int M;               // number of type slots (max id + 1)
  int nplates;
  PlateBox plate[kMaxPlates];
};

// code of component `comp` (0..5 = Ex Ey Ez Hx Hy Hz) at (i, j, k)
__device__ __forceinline__ uint32_t material_code(const MatBuild& b, int comp, int i, int j, int k) {
  const int nx = b.nx, ny = b.ny, nz = b.nz;
  const uint32_t M = (uint32_t)b.M;
  auto at = [&](int a, int c, int d) -> uint32_t { return b.mat[((long long)a * ny + c) * nz + d]; };
  if (comp < 3) {
    const uint32_t fill = M * M * M * M;
    uint32_t code = fill;
    if (comp == 0 && j >= 1 && j < ny && k >= 1 && k < nz)
      code = at(i, j, k) + M * (at(i, j - 1, k) + M * (at(i, j, k - 1) + M * at(i, j - 1, k - 1)));
    else if (comp == 1 && i >= 1 && i < nx && k >= 1 && k < nz)
      code = at(i, j, k) + M * (at(i - 1, j, k) + M * (at(i, j, k - 1) + M * at(i - 1, j, k - 1)));
    else if (comp == 2 && i >= 1 && i < nx && j >= 1 && j < ny)
      code = at(i, j, k) + M * (at(i - 1, j, k) + M * (at(i, j - 1, k) + M * at(i - 1, j - 1, k)));
    int sid = -1;
    for (int q = 0; q < b.nplates; q++) {
      const PlateBox& p = b.plate[q];
      if (p.comp == comp && i >= p.i0 && i <= p.i1 && j >= p.j0 && j <= p.j1 && k >= p.k0 && k <= p.k1)
        sid = p.sigma_id;
    }
    return code + (uint32_t)(sid + 1) * (fill + 1);
  }
  const uint32_t fill = M * M;
  if (comp == 3 && i >= 1 && i < nx) return at(i, j, k) + M * at(i - 1, j, k);
  if (comp == 4 && j >= 1 && j < ny) return at(i, j, k) + M * at(i, j - 1, k);
  if (comp == 5 && k >= 1 && k < nz) return at(i, j, k) + M * at(i, j, k - 1);
  return fill;
}

// component extents, API order Ex Ey Ez Hx Hy Hz
__device__ __forceinline__ void comp_extent(const MatBuild& b, int comp, int& ni, int& nj, int& nk) {
  const int nx = b.nx, ny = b.ny, nz = b.nz;
  ni = (comp == 0 || comp == 4 || comp == 5) ? nx : nx + 1;
  nj = (comp == 1 || comp == 3 || comp == 5) ? ny : ny + 1;
  nk = (comp == 2 || comp == 3 || comp == 4) ? nz : nz + 1;
}

__global__ void __launch_bounds__(256) k_material_mark(MatBuild b, int comp, uint8_t* present) {
  int ni, nj, nk;
  comp_extent(b, comp, ni, nj, nk);
  const long long n = (long long)ni * nj * nk;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % nk), j = (int)((t / nk) % nj), i = (int)(t / ((long long)nj * nk));
    present[material_code(b, comp, i, j, k)] = 1;  // every writer stores the same value
  }
}

__global__ void __launch_bounds__(256) k_material_ids(MatBuild b, int comp, const uint8_t* code_to_row, uint8_t* ids) {
  int ni, nj, nk;
  comp_extent(b, comp, ni, nj, nk);
  const long long n = (long long)ni * nj * nk;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % nk), j = (int)((t / nk) % nj), i = (int)(t / ((long long)nj * nk));
    ids[t] = code_to_row[material_code(b, comp, i, j, k)];
  }
}

// FP64 per-cell coefficients (the drop-in path built on the device): each
// cell of component `comp` takes the FP64 triple of its code's row, computed
// on the host with the reference's formulas (coefficients.js:22-116); out[w]
// is coefficient array 3 * comp + w.
__global__ void __launch_bounds__(256) k_material_coef(MatBuild b, int comp, const int* code_to_row,
                                                       const double* rows, double* out0, double* out1, double* out2) {
  int ni, nj, nk;
  comp_extent(b, comp, ni, nj, nk);
  const long long n = (long long)ni * nj * nk;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % nk), j = (int)((t / nk) % nj), i = (int)(t / ((long long)nj * nk));
    const long long r = code_to_row[material_code(b, comp, i, j, k)];
    out0[t] = rows[3 * r];
    out1[t] = rows[3 * r + 1];
    out2[t] = rows[3 * r + 2];
  }
}

// The CPML band of one face on one per-cell FP64 coefficient array (an array
// of extent ni x nj x nk; the band is [st, st + nc) along `axis`), as
// cpml.js:212-243 does it: CPsi (the slot's array, C order over the band) is
// the coefficient times the cell size, taken before the coefficient is divided
// by kappa of its band cell.
__global__ void __launch_bounds__(256) k_cpml_band(double* coef, int ni, int nj, int nk, int axis, int st, int nc,
                                                   double cell, const double* kappa, double* cpsi) {
  const int bi = axis == 0 ? nc : ni, bj = axis == 1 ? nc : nj, bk = axis == 2 ? nc : nk;
  const long long n = (long long)bi * bj * bk;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t % bk), b = (int)((t / bk) % bj), a = (int)(t / ((long long)bj * bk));
    const int i = a + (axis == 0 ? st : 0), j = b + (axis == 1 ? st : 0), k = c + (axis == 2 ? st : 0);
    const long long idx = ((long long)i * nj + j) * nk + k;
    const double v = coef[idx];
    cpsi[t] = __dmul_rn(v, cell);
    coef[idx] = __ddiv_rn(v, kappa[axis == 0 ? a : (axis == 1 ? b : c)]);
  }
}

// Source cells of an FP64 problem: their coefficient triples replace the
// material ones (coefficients.js:158-207).  One thread, in list order, so a
// repeated index keeps its last triple as the reference's assignment does.
__global__ void k_coef_override(double* out0, double* out1, double* out2, const int* idx, const double* trip, int n) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int q = 0; q < n; q++) {
    out0[idx[q]] = trip[3 * q];
    out1[idx[q]] = trip[3 * q + 1];
    out2[idx[q]] = trip[3 * q + 2];
  }
}

}  // namespace fdtd
