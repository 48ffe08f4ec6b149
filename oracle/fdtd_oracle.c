/*
 * fdtd_oracle.c -- CPU FP64 restatement of the MGALIKE/special-topics FDTD
 * time-step loop, used ONLY as test infrastructure: the parity checker for the
 * CUDA engine and the timed CPU baseline.  Nothing in the shipped library links
 * or calls this file.
 *
 * Every function follows one reference function statement by statement, in the
 * same loop order and with the same expression evaluation order, so that a
 * build with -ffp-contract=off reproduces the reference's Float64 arithmetic
 * bit for bit (up to the last-ulp behaviour of exp/pow/cos/sin, which the
 * reference takes from V8 and this file from the C library).
 *
 *   setup      js_fdtd/src/grid.js:16-187          buildGrid
 *              js_fdtd/src/materials.js:21-68       buildMaterialGrid
 *              js_fdtd/src/materials.js:87-238      computeMaterialComponents
 *              js_fdtd/src/materials.js:253-332     applyPECPlates
 *              js_fdtd/src/coefficients.js:22-116   computeGeneralCoefficients
 *              js_fdtd/src/cpml.js:25-448           initCPML (+ kappa division)
 *              js_fdtd/src/sources.js:16-145        initWaveforms / initVoltageSources
 *              js_fdtd/src/coefficients.js:136-207  applyLumpedElementCoefficients (voltage sources)
 *              js_fdtd/src/sampling.js:81-136       initSampledVoltages / initSampledCurrents
 *              js_fdtd/src/farfield.js:28-78        initFarfield
 *   per step   js_fdtd/assembly/fdtd_kernels.ts:20-114   updateH
 *              js_fdtd/src/cpml.js:456-724               updateMagneticCPML
 *              js_fdtd/src/sampling.js:204-245           captureSampledCurrents
 *              js_fdtd/assembly/fdtd_kernels.ts:116-210  updateE
 *              js_fdtd/src/cpml.js:727-1003              updateElectricCPML
 *              js_fdtd/src/sources.js:271-288            injectVoltageSources
 *              js_fdtd/src/sampling.js:295-307           captureSampledVoltages
 *              js_fdtd/src/farfield.js:90-248            accumulateFarfieldDFT
 *              (order: js_fdtd/src/fdtdSolver.js:84-118, CONTRACT.md:61-96)
 *   post       js_fdtd/src/dft.js:17-38             timeToFreqDomain
 *              js_fdtd/src/sparameters.js:118-196   computePortWaves / computeSMatrix
 *              js_fdtd/src/farfield.js:257-607      calcRadiatedPower / calcDirectivity
 *
 * Memory: the six field arrays live in ONE allocation in the order
 * Hx,Hy,Hz,Ex,Ey,Ez, exactly like the reference's shared WebAssembly.Memory
 * (grid.js:136-141).  updateE's i = nx planes of Ey/Ez read Hz/Hy one plane past
 * their end (fdtd_kernels.ts:159-163,185-188 with the partition end nxp1 from
 * fdtdWorker.js:22-30); in the reference those reads land in the next array of
 * the shared memory, and the same layout here makes them land in the same
 * place.  With the reference's usual worker count the thread that owns the
 * i = nx plane starts its Ey rows while worker 0 is still rewriting Ex(i=0),
 * the very values those out-of-range Hz reads return, so the reference itself
 * reads a run-dependent mix of pre- and post-update Ex(i=0).  This oracle reads
 * the post-update values (serial order) by default; ofd_set_edge_read(1)
 * selects the pre-update values, and the two runs bracket the reference's
 * output (the golden-file test checks that they do).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EPS0 8.854187817e-12
#define C0 2.99792458e8
#define ETA0 376.73031346177066

static const double MU0 = 4 * M_PI * 1e-7; /* constants.js:5 / cpml.js:144 */

/* ------------------------------------------------------------------------- */
/* Scenario description passed in by the ctypes wrapper (oracle/oracle.py).  */
/* ------------------------------------------------------------------------- */
typedef struct {
  double dx, dy, dz, courant;
  int nsteps;
  int is_cpml[6]; /* xn xp yn yp zn zp */
  int air[6];
  int ncpml[6];
  double cpml_order, sigma_factor, kappa_max, alpha_min, alpha_max;
  int n_mat;    const double* mat;    /* [n][4] eps_r mu_r sigma_e sigma_m           */
  int n_brick;  const double* brick;  /* [n][7] min_x min_y min_z max_x max_y max_z t */
  int n_sphere; const double* sphere; /* [n][5] cx cy cz r t                         */
  int n_wave;   const double* wave;   /* [n][4] kind p0 p1 p2                        */
  int n_vs;     const double* vs;     /* [n][11] min(3) max(3) axis sign R mag wave  */
  int n_sv;     const double* sv;     /* [n][8]  min(3) max(3) axis sign             */
  int n_si;     const double* si;     /* [n][8]  min(3) max(3) axis sign             */
  int n_ff;     const double* ff_freq;
  int nc_ff;
} ofd_scn;

typedef struct {
  int nc;
  int axis, ascending;
  double *b_e, *a_e, *b_m, *a_m, *kappa_e, *kappa_m;
  /* magnetic psi/cpsi slots 0,1 and electric slots 2,3 (component order below) */
  double *psi[4], *cpsi[4];
  long npsi[4];
  int m_start, e_start;
} ofd_face;

typedef struct {
  int n; /* number of gap cells */
  int axis;
  int32_t* fi;
  double* cs;   /* Cexs / Ceys / Cezs */
  double* vpe;  /* voltage_per_e_field[nsteps] */
  double resistance_per_component;
} ofd_vsrc;

typedef struct {
  int axis, sign;
  int is, js, ks, ie, je, ke;
  int nfi;
  int32_t* fi;
  double Csvf;
  double* val;
} ofd_probe;

typedef struct {
  int nx, ny, nz, nxp1, nyp1, nzp1;
  double dx, dy, dz, dt;
  double min_x, min_y, min_z, max_x, max_y, max_z;
  int nsteps, ts;
  long nhx, nhy, nhz, nex, ney, nez;
  double* fields; /* Hx Hy Hz Ex Ey Ez, contiguous */
  double *Hx, *Hy, *Hz, *Ex, *Ey, *Ez;
  double* coef;   /* 18 arrays, order below */
  double *Cexe, *Cexhz, *Cexhy, *Ceye, *Ceyhx, *Ceyhz, *Ceze, *Cezhy, *Cezhx;
  double *Chxh, *Chxez, *Chxey, *Chyh, *Chyex, *Chyez, *Chzh, *Chzey, *Chzex;
  /* material components (kept for inspection) */
  double *eps_r_x, *eps_r_y, *eps_r_z, *mu_r_x, *mu_r_y, *mu_r_z;
  double *sigma_e_x, *sigma_e_y, *sigma_e_z, *sigma_m_x, *sigma_m_y, *sigma_m_z;
  uint8_t* mat;
  ofd_face face[6];
  int has_face[6];
  int n_vs; ofd_vsrc* vs;
  int n_sv; ofd_probe* sv;
  int n_si; ofd_probe* si;
  double** waves; int n_wave;
  /* far field */
  int nFreq, li, lj, lk, ui, uj, uk, ni_ff, nj_ff, nk_ff;
  long sz_x, sz_y, sz_z;
  double* ffreq;
  double* w;
  double* ffacc; /* 24 arrays x {re,im}, order FF_NAMES */
  double* ffp[24][2];
} ofd_state;

static const char* FF_NAMES[24] = {
    "cjyxp", "cjzxp", "cjyxn", "cjzxn", "cjxyp", "cjzyp", "cjxyn", "cjzyn",
    "cjxzp", "cjyzp", "cjxzn", "cjyzn", "cmyxp", "cmzxp", "cmyxn", "cmzxn",
    "cmxyp", "cmzyp", "cmxyn", "cmzyn", "cmxzp", "cmyzp", "cmxzn", "cmyzn"};
enum {
  CJYXP, CJZXP, CJYXN, CJZXN, CJXYP, CJZYP, CJXYN, CJZYN, CJXZP, CJYZP, CJXZN, CJYZN,
  CMYXP, CMZXP, CMYXN, CMZXN, CMXYP, CMZYP, CMXYN, CMZYN, CMXZP, CMYZP, CMXZN, CMYZN
};

/* Math.round: nearest integer, ties toward +infinity. */
static int js_round(double x) {
  double f = floor(x);
  return (int)((x - f >= 0.5) ? f + 1.0 : f);
}

static void* xcalloc(size_t n, size_t sz) {
  void* p = calloc(n ? n : 1, sz);
  if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
  return p;
}

/* ------------------------------------------------------------------------- */
/* grid.js:16-187                                                             */
/* ------------------------------------------------------------------------- */
static void build_grid(ofd_state* g, const ofd_scn* s) {
  const double dx = s->dx, dy = s->dy, dz = s->dz;
  double min_x = INFINITY, min_y = INFINITY, min_z = INFINITY;
  double max_x = -INFINITY, max_y = -INFINITY, max_z = -INFINITY;
  for (int n = 0; n < s->n_sphere; n++) {
    const double* sp = s->sphere + 5 * n;
    min_x = fmin(min_x, sp[0] - sp[3]);
    min_y = fmin(min_y, sp[1] - sp[3]);
    min_z = fmin(min_z, sp[2] - sp[3]);
    max_x = fmax(max_x, sp[0] + sp[3]);
    max_y = fmax(max_y, sp[1] + sp[3]);
    max_z = fmax(max_z, sp[2] + sp[3]);
  }
  for (int n = 0; n < s->n_brick; n++) {
    const double* b = s->brick + 7 * n;
    min_x = fmin(min_x, b[0]);
    min_y = fmin(min_y, b[1]);
    min_z = fmin(min_z, b[2]);
    max_x = fmax(max_x, b[3]);
    max_y = fmax(max_y, b[4]);
    max_z = fmax(max_z, b[5]);
  }
  min_x -= dx * s->air[0];
  min_y -= dy * s->air[2];
  min_z -= dz * s->air[4];
  max_x += dx * s->air[1];
  max_y += dy * s->air[3];
  max_z += dz * s->air[5];
  if (s->is_cpml[0] && s->ncpml[0] > 0) min_x -= dx * s->ncpml[0];
  if (s->is_cpml[1] && s->ncpml[1] > 0) max_x += dx * s->ncpml[1];
  if (s->is_cpml[2] && s->ncpml[2] > 0) min_y -= dy * s->ncpml[2];
  if (s->is_cpml[3] && s->ncpml[3] > 0) max_y += dy * s->ncpml[3];
  if (s->is_cpml[4] && s->ncpml[4] > 0) min_z -= dz * s->ncpml[4];
  if (s->is_cpml[5] && s->ncpml[5] > 0) max_z += dz * s->ncpml[5];

  g->nx = js_round((max_x - min_x) / dx);
  g->ny = js_round((max_y - min_y) / dy);
  g->nz = js_round((max_z - min_z) / dz);
  g->nxp1 = g->nx + 1; g->nyp1 = g->ny + 1; g->nzp1 = g->nz + 1;
  g->min_x = min_x; g->min_y = min_y; g->min_z = min_z;
  g->max_x = min_x + g->nx * dx;
  g->max_y = min_y + g->ny * dy;
  g->max_z = min_z + g->nz * dz;
  g->dx = dx; g->dy = dy; g->dz = dz;
  g->dt = s->courant / (C0 * sqrt(1 / (dx * dx) + 1 / (dy * dy) + 1 / (dz * dz)));

  const long nx = g->nx, ny = g->ny, nz = g->nz, nxp1 = g->nxp1, nyp1 = g->nyp1, nzp1 = g->nzp1;
  g->nhx = nxp1 * ny * nz;
  g->nhy = nx * nyp1 * nz;
  g->nhz = nx * ny * nzp1;
  g->nex = nx * nyp1 * nzp1;
  g->ney = nxp1 * ny * nzp1;
  g->nez = nxp1 * nyp1 * nz;
  long tot = g->nhx + g->nhy + g->nhz + g->nex + g->ney + g->nez;
  /* one spare plane of slack past Ez mirrors the +100 padding pages of grid.js:123 */
  g->fields = (double*)xcalloc(tot + (size_t)nyp1 * nzp1 + 64, sizeof(double));
  g->Hx = g->fields;
  g->Hy = g->Hx + g->nhx;
  g->Hz = g->Hy + g->nhy;
  g->Ex = g->Hz + g->nhz;
  g->Ey = g->Ex + g->nex;
  g->Ez = g->Ey + g->ney;
  long ctot = 3 * (g->nex + g->ney + g->nez + g->nhx + g->nhy + g->nhz);
  g->coef = (double*)xcalloc(ctot, sizeof(double));
  double* p = g->coef;
  g->Cexe = p; p += g->nex; g->Cexhz = p; p += g->nex; g->Cexhy = p; p += g->nex;
  g->Ceye = p; p += g->ney; g->Ceyhx = p; p += g->ney; g->Ceyhz = p; p += g->ney;
  g->Ceze = p; p += g->nez; g->Cezhy = p; p += g->nez; g->Cezhx = p; p += g->nez;
  g->Chxh = p; p += g->nhx; g->Chxez = p; p += g->nhx; g->Chxey = p; p += g->nhx;
  g->Chyh = p; p += g->nhy; g->Chyex = p; p += g->nhy; g->Chyez = p; p += g->nhy;
  g->Chzh = p; p += g->nhz; g->Chzey = p; p += g->nhz; g->Chzex = p; p += g->nhz;
}

/* ------------------------------------------------------------------------- */
/* materials.js:21-332                                                        */
/* ------------------------------------------------------------------------- */
static void build_materials(ofd_state* g, const ofd_scn* s) {
  const int nx = g->nx, ny = g->ny, nz = g->nz, nxp1 = g->nxp1, nyp1 = g->nyp1, nzp1 = g->nzp1;
  const double dx = g->dx, dy = g->dy, dz = g->dz;
  uint8_t* mat = (uint8_t*)xcalloc((size_t)nx * ny * nz, 1);
  memset(mat, 1, (size_t)nx * ny * nz);
  g->mat = mat;
  for (int n = 0; n < s->n_sphere; n++) {
    const double* sp = s->sphere + 5 * n;
    const double r2 = sp[3] * sp[3];
    for (int i = 0; i < nx; i++) {
      const double cx = (i + 0.5) * dx + g->min_x;
      for (int j = 0; j < ny; j++) {
        const double cy = (j + 0.5) * dy + g->min_y;
        for (int k = 0; k < nz; k++) {
          const double cz = (k + 0.5) * dz + g->min_z;
          const double dx2 = cx - sp[0], dy2 = cy - sp[1], dz2 = cz - sp[2];
          if (dx2 * dx2 + dy2 * dy2 + dz2 * dz2 <= r2) mat[(long)i * ny * nz + j * nz + k] = (uint8_t)(int)sp[4];
        }
      }
    }
  }
  for (int n = 0; n < s->n_brick; n++) {
    const double* b = s->brick + 7 * n;
    const int blx = js_round((b[0] - g->min_x) / dx), bly = js_round((b[1] - g->min_y) / dy),
              blz = js_round((b[2] - g->min_z) / dz);
    const int bux = js_round((b[3] - g->min_x) / dx), buy = js_round((b[4] - g->min_y) / dy),
              buz = js_round((b[5] - g->min_z) / dz);
    for (int i = blx; i < bux; i++) {
      if (i < 0 || i >= nx) continue;
      for (int j = bly; j < buy; j++) {
        if (j < 0 || j >= ny) continue;
        for (int k = blz; k < buz; k++) {
          if (k < 0 || k >= nz) continue;
          mat[(long)i * ny * nz + j * nz + k] = (uint8_t)(int)b[6];
        }
      }
    }
  }

  const int nmt = s->n_mat;
  double* t_eps = (double*)xcalloc(nmt + 1, sizeof(double));
  double* t_mu = (double*)xcalloc(nmt + 1, sizeof(double));
  double* t_se = (double*)xcalloc(nmt + 1, sizeof(double));
  double* t_sm = (double*)xcalloc(nmt + 1, sizeof(double));
  for (int m = 0; m < nmt; m++) {
    const double* mt = s->mat + 4 * m;
    t_eps[m + 1] = mt[0];
    t_mu[m + 1] = (mt[1] != 0 && mt[1] == mt[1]) ? mt[1] : 1e-20;
    t_se[m + 1] = mt[2];
    t_sm[m + 1] = (mt[3] != 0 && mt[3] == mt[3]) ? mt[3] : 1e-20;
  }
#define MT(i, j, k) mat[(long)((i) < 0 ? 0 : ((i) > nx - 1 ? nx - 1 : (i))) * ny * nz + \
                        (long)((j) < 0 ? 0 : ((j) > ny - 1 ? ny - 1 : (j))) * nz +   \
                        ((k) < 0 ? 0 : ((k) > nz - 1 ? nz - 1 : (k)))]
  const long nex = g->nex, ney = g->ney, nez = g->nez, nhx = g->nhx, nhy = g->nhy, nhz = g->nhz;
  g->eps_r_x = (double*)xcalloc(nex, 8); g->eps_r_y = (double*)xcalloc(ney, 8); g->eps_r_z = (double*)xcalloc(nez, 8);
  g->mu_r_x = (double*)xcalloc(nhx, 8); g->mu_r_y = (double*)xcalloc(nhy, 8); g->mu_r_z = (double*)xcalloc(nhz, 8);
  g->sigma_e_x = (double*)xcalloc(nex, 8); g->sigma_e_y = (double*)xcalloc(ney, 8); g->sigma_e_z = (double*)xcalloc(nez, 8);
  g->sigma_m_x = (double*)xcalloc(nhx, 8); g->sigma_m_y = (double*)xcalloc(nhy, 8); g->sigma_m_z = (double*)xcalloc(nhz, 8);
  for (long n = 0; n < nex; n++) g->eps_r_x[n] = 1.0;
  for (long n = 0; n < ney; n++) g->eps_r_y[n] = 1.0;
  for (long n = 0; n < nez; n++) g->eps_r_z[n] = 1.0;
  for (long n = 0; n < nhx; n++) g->mu_r_x[n] = 1.0;
  for (long n = 0; n < nhy; n++) g->mu_r_y[n] = 1.0;
  for (long n = 0; n < nhz; n++) g->mu_r_z[n] = 1.0;

  for (int i = 0; i < nx; i++)
    for (int j = 1; j < ny; j++)
      for (int k = 1; k < nz; k++) {
        const long idx = (long)i * nyp1 * nzp1 + j * nzp1 + k;
        const int m1 = MT(i, j, k), m2 = MT(i, j - 1, k), m3 = MT(i, j, k - 1), m4 = MT(i, j - 1, k - 1);
        g->eps_r_x[idx] = 0.25 * (t_eps[m1] + t_eps[m2] + t_eps[m3] + t_eps[m4]);
        g->sigma_e_x[idx] = 0.25 * (t_se[m1] + t_se[m2] + t_se[m3] + t_se[m4]);
      }
  for (int i = 1; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 1; k < nz; k++) {
        const long idx = (long)i * ny * nzp1 + j * nzp1 + k;
        const int m1 = MT(i, j, k), m2 = MT(i - 1, j, k), m3 = MT(i, j, k - 1), m4 = MT(i - 1, j, k - 1);
        g->eps_r_y[idx] = 0.25 * (t_eps[m1] + t_eps[m2] + t_eps[m3] + t_eps[m4]);
        g->sigma_e_y[idx] = 0.25 * (t_se[m1] + t_se[m2] + t_se[m3] + t_se[m4]);
      }
  for (int i = 1; i < nx; i++)
    for (int j = 1; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        const long idx = (long)i * nyp1 * nz + j * nz + k;
        const int m1 = MT(i, j, k), m2 = MT(i - 1, j, k), m3 = MT(i, j - 1, k), m4 = MT(i - 1, j - 1, k);
        g->eps_r_z[idx] = 0.25 * (t_eps[m1] + t_eps[m2] + t_eps[m3] + t_eps[m4]);
        g->sigma_e_z[idx] = 0.25 * (t_se[m1] + t_se[m2] + t_se[m3] + t_se[m4]);
      }
  for (int i = 1; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        const long idx = (long)i * ny * nz + j * nz + k;
        const double mu1 = t_mu[MT(i, j, k)], mu2 = t_mu[MT(i - 1, j, k)];
        g->mu_r_x[idx] = 2 * mu1 * mu2 / (mu1 + mu2);
        const double sm1 = t_sm[MT(i, j, k)], sm2 = t_sm[MT(i - 1, j, k)];
        g->sigma_m_x[idx] = 2 * sm1 * sm2 / (sm1 + sm2);
      }
  for (int i = 0; i < nx; i++)
    for (int j = 1; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        const long idx = (long)i * nyp1 * nz + j * nz + k;
        const double mu1 = t_mu[MT(i, j, k)], mu2 = t_mu[MT(i, j - 1, k)];
        g->mu_r_y[idx] = 2 * mu1 * mu2 / (mu1 + mu2);
        const double sm1 = t_sm[MT(i, j, k)], sm2 = t_sm[MT(i, j - 1, k)];
        g->sigma_m_y[idx] = 2 * sm1 * sm2 / (sm1 + sm2);
      }
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 1; k < nz; k++) {
        const long idx = (long)i * ny * nzp1 + j * nzp1 + k;
        const double mu1 = t_mu[MT(i, j, k)], mu2 = t_mu[MT(i, j, k - 1)];
        g->mu_r_z[idx] = 2 * mu1 * mu2 / (mu1 + mu2);
        const double sm1 = t_sm[MT(i, j, k)], sm2 = t_sm[MT(i, j, k - 1)];
        g->sigma_m_z[idx] = 2 * sm1 * sm2 / (sm1 + sm2);
      }
#undef MT

  /* applyPECPlates: materials.js:253-332 */
  for (int n = 0; n < s->n_brick; n++) {
    const double* b = s->brick + 7 * n;
    const int t = (int)b[6];
    if (t < 1 || t > nmt) continue;
    const double sigma_pec = s->mat[4 * (t - 1) + 2];
    if (sigma_pec == 0) continue;
    const int blx = js_round((b[0] - g->min_x) / dx) + 1, bly = js_round((b[1] - g->min_y) / dy) + 1,
              blz = js_round((b[2] - g->min_z) / dz) + 1;
    const int bux = js_round((b[3] - g->min_x) / dx) + 1, buy = js_round((b[4] - g->min_y) / dy) + 1,
              buz = js_round((b[5] - g->min_z) / dz) + 1;
    if (blx == bux) {
      const int i = blx - 1;
      if (i >= 0 && i < nxp1) {
        for (int j = bly - 1; j < buy - 1; j++)
          for (int k = blz - 1; k < buz; k++)
            if (j >= 0 && j < ny && k >= 0 && k < nzp1) g->sigma_e_y[(long)i * ny * nzp1 + j * nzp1 + k] = sigma_pec;
        for (int j = bly - 1; j < buy; j++)
          for (int k = blz - 1; k < buz - 1; k++)
            if (j >= 0 && j < nyp1 && k >= 0 && k < nz) g->sigma_e_z[(long)i * nyp1 * nz + j * nz + k] = sigma_pec;
      }
    }
    if (bly == buy) {
      const int j = bly - 1;
      if (j >= 0 && j < nyp1) {
        for (int i = blx - 1; i < bux - 1; i++)
          for (int k = blz - 1; k < buz; k++)
            if (i >= 0 && i < nx && k >= 0 && k < nzp1) g->sigma_e_x[(long)i * nyp1 * nzp1 + j * nzp1 + k] = sigma_pec;
        for (int i = blx - 1; i < bux; i++)
          for (int k = blz - 1; k < buz - 1; k++)
            if (i >= 0 && i < nxp1 && k >= 0 && k < nz) g->sigma_e_z[(long)i * nyp1 * nz + j * nz + k] = sigma_pec;
      }
    }
    if (blz == buz) {
      const int k = blz - 1;
      if (k >= 0 && k < nzp1) {
        for (int i = blx - 1; i < bux - 1; i++)
          for (int j = bly - 1; j < buy; j++)
            if (i >= 0 && i < nx && j >= 0 && j < nyp1) g->sigma_e_x[(long)i * nyp1 * nzp1 + j * nzp1 + k] = sigma_pec;
        for (int i = blx - 1; i < bux; i++)
          for (int j = bly - 1; j < buy - 1; j++)
            if (i >= 0 && i < nxp1 && j >= 0 && j < ny) g->sigma_e_y[(long)i * ny * nzp1 + j * nzp1 + k] = sigma_pec;
      }
    }
  }
  free(t_eps); free(t_mu); free(t_se); free(t_sm);
}

/* ------------------------------------------------------------------------- */
/* coefficients.js:22-116                                                     */
/* ------------------------------------------------------------------------- */
static void general_coefficients(ofd_state* g) {
  const double dt = g->dt;
  const double two_dt_dy = 2 * dt / g->dy, two_dt_dz = 2 * dt / g->dz, two_dt_dx = 2 * dt / g->dx;
  for (long n = 0; n < g->nex; n++) {
    const double denom = 2 * g->eps_r_x[n] * EPS0 + dt * g->sigma_e_x[n];
    g->Cexe[n] = (2 * g->eps_r_x[n] * EPS0 - dt * g->sigma_e_x[n]) / denom;
    g->Cexhz[n] = two_dt_dy / denom;
    g->Cexhy[n] = -two_dt_dz / denom;
  }
  for (long n = 0; n < g->ney; n++) {
    const double denom = 2 * g->eps_r_y[n] * EPS0 + dt * g->sigma_e_y[n];
    g->Ceye[n] = (2 * g->eps_r_y[n] * EPS0 - dt * g->sigma_e_y[n]) / denom;
    g->Ceyhx[n] = two_dt_dz / denom;
    g->Ceyhz[n] = -two_dt_dx / denom;
  }
  for (long n = 0; n < g->nez; n++) {
    const double denom = 2 * g->eps_r_z[n] * EPS0 + dt * g->sigma_e_z[n];
    g->Ceze[n] = (2 * g->eps_r_z[n] * EPS0 - dt * g->sigma_e_z[n]) / denom;
    g->Cezhy[n] = two_dt_dx / denom;
    g->Cezhx[n] = -two_dt_dy / denom;
  }
  for (long n = 0; n < g->nhx; n++) {
    const double denom = 2 * g->mu_r_x[n] * MU0 + dt * g->sigma_m_x[n];
    g->Chxh[n] = (2 * g->mu_r_x[n] * MU0 - dt * g->sigma_m_x[n]) / denom;
    g->Chxez[n] = -two_dt_dy / denom;
    g->Chxey[n] = two_dt_dz / denom;
  }
  for (long n = 0; n < g->nhy; n++) {
    const double denom = 2 * g->mu_r_y[n] * MU0 + dt * g->sigma_m_y[n];
    g->Chyh[n] = (2 * g->mu_r_y[n] * MU0 - dt * g->sigma_m_y[n]) / denom;
    g->Chyex[n] = -two_dt_dz / denom;
    g->Chyez[n] = two_dt_dx / denom;
  }
  for (long n = 0; n < g->nhz; n++) {
    const double denom = 2 * g->mu_r_z[n] * MU0 + dt * g->sigma_m_z[n];
    g->Chzh[n] = (2 * g->mu_r_z[n] * MU0 - dt * g->sigma_m_z[n]) / denom;
    g->Chzey[n] = -two_dt_dx / denom;
    g->Chzex[n] = two_dt_dy / denom;
  }
}

/* ------------------------------------------------------------------------- */
/* cpml.js:100-141 (_cpml1D)                                                  */
/* ------------------------------------------------------------------------- */
static void cpml_1d(ofd_face* f, double cell, double dt, double p_order, double sigma_ratio,
                    double kappa_max, double alpha_min, double alpha_max, int ascending) {
  const int nc = f->nc;
  const double sigma_max = sigma_ratio * (p_order + 1) / (150 * M_PI * cell);
  f->b_e = (double*)xcalloc(nc, 8); f->a_e = (double*)xcalloc(nc, 8);
  f->b_m = (double*)xcalloc(nc, 8); f->a_m = (double*)xcalloc(nc, 8);
  f->kappa_e = (double*)xcalloc(nc, 8); f->kappa_m = (double*)xcalloc(nc, 8);
  for (int ci = 0; ci < nc; ci++) {
    const double rho_e = ascending ? (ci + 1 - 0.75) / nc : (nc - ci - 0.75) / nc;
    const double rho_m = ascending ? (ci + 1 - 0.25) / nc : (nc - ci - 0.25) / nc;
    const double se = sigma_max * pow(rho_e, p_order);
    const double sm = (MU0 / EPS0) * sigma_max * pow(rho_m, p_order);
    const double ke = 1 + (kappa_max - 1) * pow(rho_e, p_order);
    const double km = 1 + (kappa_max - 1) * pow(rho_m, p_order);
    const double ae = alpha_min + (alpha_max - alpha_min) * (1 - rho_e);
    const double am = (MU0 / EPS0) * (alpha_min + (alpha_max - alpha_min) * (1 - rho_m));
    f->b_e[ci] = exp(-(dt / EPS0) * (se / ke + ae));
    f->a_e[ci] = (1 / cell) * (f->b_e[ci] - 1) * se / (ke * (se + ke * ae));
    f->b_m[ci] = exp(-(dt / MU0) * (sm / km + am));
    f->a_m[ci] = (1 / cell) * (f->b_m[ci] - 1) * sm / (km * (sm + km * am));
    f->kappa_e[ci] = ke;
    f->kappa_m[ci] = km;
  }
}

/*
 * cpml.js:147-448.  Slot convention (same meaning for all axes):
 *   x face: 0=hyx (nc,nyp1,nz) 1=hzx (nc,ny,nzp1) 2=eyx (nc,ny,nzp1) 3=ezx (nc,nyp1,nz)
 *   y face: 0=hxy (nxp1,nc,nz) 1=hzy (nx,nc,nzp1) 2=ezy (nxp1,nc,nz) 3=exy (nx,nc,nzp1)
 *   z face: 0=hxz (nxp1,ny,nc) 1=hyz (nx,nyp1,nc) 2=exz (nx,nyp1,nc) 3=eyz (nxp1,ny,nc)
 */
static void init_face(ofd_state* g, const ofd_scn* s, int fid) {
  ofd_face* f = &g->face[fid];
  const int axis = fid / 2, ascending = fid & 1;
  const int nc = s->ncpml[fid];
  const long nx = g->nx, ny = g->ny, nz = g->nz, nxp1 = g->nxp1, nyp1 = g->nyp1, nzp1 = g->nzp1;
  f->nc = nc; f->axis = axis; f->ascending = ascending;
  const double cell = axis == 0 ? g->dx : (axis == 1 ? g->dy : g->dz);
  cpml_1d(f, cell, g->dt, s->cpml_order, s->sigma_factor, s->kappa_max, s->alpha_min, s->alpha_max, ascending);
  if (axis == 0) {
    f->npsi[0] = nc * nyp1 * nz; f->npsi[1] = nc * ny * nzp1; f->npsi[2] = nc * ny * nzp1; f->npsi[3] = nc * nyp1 * nz;
  } else if (axis == 1) {
    f->npsi[0] = nxp1 * nc * nz; f->npsi[1] = nx * nc * nzp1; f->npsi[2] = nxp1 * nc * nz; f->npsi[3] = nx * nc * nzp1;
  } else {
    f->npsi[0] = nxp1 * ny * nc; f->npsi[1] = nx * nyp1 * nc; f->npsi[2] = nx * nyp1 * nc; f->npsi[3] = nxp1 * ny * nc;
  }
  for (int q = 0; q < 4; q++) {
    f->psi[q] = (double*)xcalloc(f->npsi[q], 8);
    f->cpsi[q] = (double*)xcalloc(f->npsi[q], 8);
  }
  if (axis == 0) {
    const int n_st = ascending ? (int)(nx - nc) : 0;
    f->m_start = n_st;
    f->e_start = ascending ? (int)(nx - nc) : 1;
    for (int ci = 0; ci < nc; ci++) {
      const long i_h = n_st + ci;
      const long i_e = ascending ? n_st + ci : ci + 1;
      for (long j = 0; j < nyp1; j++)
        for (long k = 0; k < nz; k++) f->cpsi[0][ci * nyp1 * nz + j * nz + k] = g->Chyez[i_h * nyp1 * nz + j * nz + k] * g->dx;
      for (long j = 0; j < ny; j++)
        for (long k = 0; k < nzp1; k++) f->cpsi[1][ci * ny * nzp1 + j * nzp1 + k] = g->Chzey[i_h * ny * nzp1 + j * nzp1 + k] * g->dx;
      if (i_e >= 0 && i_e < nxp1) {
        for (long j = 0; j < ny; j++)
          for (long k = 0; k < nzp1; k++) f->cpsi[2][ci * ny * nzp1 + j * nzp1 + k] = g->Ceyhz[i_e * ny * nzp1 + j * nzp1 + k] * g->dx;
        for (long j = 0; j < nyp1; j++)
          for (long k = 0; k < nz; k++) f->cpsi[3][ci * nyp1 * nz + j * nz + k] = g->Cezhy[i_e * nyp1 * nz + j * nz + k] * g->dx;
      }
    }
    for (int ci = 0; ci < nc; ci++) {
      const long i_h = n_st + ci;
      const long i_e = ascending ? (nx - nc + ci) : (ci + 1);
      const double ke = f->kappa_e[ci], km = f->kappa_m[ci];
      for (long j = 0; j < nyp1; j++)
        for (long k = 0; k < nz; k++) g->Chyez[i_h * nyp1 * nz + j * nz + k] /= km;
      for (long j = 0; j < ny; j++)
        for (long k = 0; k < nzp1; k++) g->Chzey[i_h * ny * nzp1 + j * nzp1 + k] /= km;
      if (i_e >= 0 && i_e < nxp1) {
        for (long j = 0; j < ny; j++)
          for (long k = 0; k < nzp1; k++) g->Ceyhz[i_e * ny * nzp1 + j * nzp1 + k] /= ke;
        for (long j = 0; j < nyp1; j++)
          for (long k = 0; k < nz; k++) g->Cezhy[i_e * nyp1 * nz + j * nz + k] /= ke;
      }
    }
  } else if (axis == 1) {
    const int n_st = ascending ? (int)(ny - nc) : 0;
    f->m_start = n_st;
    f->e_start = ascending ? (int)(ny - nc) : 1;
    for (int ci = 0; ci < nc; ci++) {
      const long j_h = n_st + ci;
      const long j_e = ascending ? (ny - nc + ci) : (ci + 1);
      for (long i = 0; i < nxp1; i++)
        for (long k = 0; k < nz; k++) f->cpsi[0][i * nc * nz + ci * nz + k] = g->Chxez[i * ny * nz + j_h * nz + k] * g->dy;
      for (long i = 0; i < nx; i++)
        for (long k = 0; k < nzp1; k++) f->cpsi[1][i * nc * nzp1 + ci * nzp1 + k] = g->Chzex[i * ny * nzp1 + j_h * nzp1 + k] * g->dy;
      if (j_e >= 0 && j_e < nyp1) {
        for (long i = 0; i < nxp1; i++)
          for (long k = 0; k < nz; k++) f->cpsi[2][i * nc * nz + ci * nz + k] = g->Cezhx[i * nyp1 * nz + j_e * nz + k] * g->dy;
        for (long i = 0; i < nx; i++)
          for (long k = 0; k < nzp1; k++) f->cpsi[3][i * nc * nzp1 + ci * nzp1 + k] = g->Cexhz[i * nyp1 * nzp1 + j_e * nzp1 + k] * g->dy;
      }
    }
    for (int ci = 0; ci < nc; ci++) {
      const long j_h = n_st + ci;
      const long j_e = ascending ? (ny - nc + ci) : (ci + 1);
      const double ke = f->kappa_e[ci], km = f->kappa_m[ci];
      for (long i = 0; i < nxp1; i++)
        for (long k = 0; k < nz; k++) g->Chxez[i * ny * nz + j_h * nz + k] /= km;
      for (long i = 0; i < nx; i++)
        for (long k = 0; k < nzp1; k++) g->Chzex[i * ny * nzp1 + j_h * nzp1 + k] /= km;
      if (j_e >= 0 && j_e < nyp1) {
        for (long i = 0; i < nxp1; i++)
          for (long k = 0; k < nz; k++) g->Cezhx[i * nyp1 * nz + j_e * nz + k] /= ke;
        for (long i = 0; i < nx; i++)
          for (long k = 0; k < nzp1; k++) g->Cexhz[i * nyp1 * nzp1 + j_e * nzp1 + k] /= ke;
      }
    }
  } else {
    const int n_st = ascending ? (int)(nz - nc) : 0;
    f->m_start = n_st;
    f->e_start = ascending ? (int)(nz - nc) : 1;
    for (int ci = 0; ci < nc; ci++) {
      const long k_h = n_st + ci;
      const long k_e = ascending ? (nz - nc + ci) : (ci + 1);
      for (long i = 0; i < nxp1; i++)
        for (long j = 0; j < ny; j++) f->cpsi[0][i * ny * nc + j * nc + ci] = g->Chxey[i * ny * nz + j * nz + k_h] * g->dz;
      for (long i = 0; i < nx; i++)
        for (long j = 0; j < nyp1; j++) f->cpsi[1][i * nyp1 * nc + j * nc + ci] = g->Chyex[i * nyp1 * nz + j * nz + k_h] * g->dz;
      if (k_e >= 0 && k_e < nzp1) {
        for (long i = 0; i < nx; i++)
          for (long j = 0; j < nyp1; j++) f->cpsi[2][i * nyp1 * nc + j * nc + ci] = g->Cexhy[i * nyp1 * nzp1 + j * nzp1 + k_e] * g->dz;
        for (long i = 0; i < nxp1; i++)
          for (long j = 0; j < ny; j++) f->cpsi[3][i * ny * nc + j * nc + ci] = g->Ceyhx[i * ny * nzp1 + j * nzp1 + k_e] * g->dz;
      }
    }
    for (int ci = 0; ci < nc; ci++) {
      const long k_h = n_st + ci;
      const long k_e = ascending ? (nz - nc + ci) : (ci + 1);
      const double ke = f->kappa_e[ci], km = f->kappa_m[ci];
      for (long i = 0; i < nxp1; i++)
        for (long j = 0; j < ny; j++) g->Chxey[i * ny * nz + j * nz + k_h] /= km;
      for (long i = 0; i < nx; i++)
        for (long j = 0; j < nyp1; j++) g->Chyex[i * nyp1 * nz + j * nz + k_h] /= km;
      if (k_e >= 0 && k_e < nzp1) {
        for (long i = 0; i < nx; i++)
          for (long j = 0; j < nyp1; j++) g->Cexhy[i * nyp1 * nzp1 + j * nzp1 + k_e] /= ke;
        for (long i = 0; i < nxp1; i++)
          for (long j = 0; j < ny; j++) g->Ceyhx[i * ny * nzp1 + j * nzp1 + k_e] /= ke;
      }
    }
  }
}

/* ------------------------------------------------------------------------- */
/* sources.js:16-94 (initWaveforms)                                           */
/* ------------------------------------------------------------------------- */
static double* make_waveform(const double* w, int N, double dt, double maxCell) {
  double* out = (double*)xcalloc(N, 8);
  const int kind = (int)w[0];
  for (int n = 0; n < N; n++) {
    const double t = (n + 0.5) * dt;
    if (kind == 0) { /* gaussian */
      const double nc = w[1];
      const double tau = (nc * maxCell) / (2 * C0);
      const double t0 = 4.5 * tau;
      const double arg = (t - t0) / tau;
      out[n] = exp(-arg * arg);
    } else if (kind == 1) { /* derivative_gaussian */
      const double nc = w[1];
      const double tau = (nc * maxCell) / (2 * C0);
      const double t0 = 4.5 * tau;
      const double scale = -sqrt(2 * M_E) / tau;
      const double dt2 = t - t0;
      const double arg = dt2 / tau;
      out[n] = scale * dt2 * exp(-arg * arg);
    } else if (kind == 2) { /* sinusoidal */
      out[n] = sin(2 * M_PI * w[1] * t);
    } else if (kind == 3) { /* unit_step */
      out[n] = (n < (int)w[1] - 1) ? 0.0 : 1.0;
    } else { /* cosine_modulated_gaussian */
      const double tau = 0.966 / w[1];
      const double t0 = 4.5 * tau;
      const double dt2 = t - t0;
      const double arg = dt2 / tau;
      out[n] = cos(2 * M_PI * w[2] * dt2) * exp(-arg * arg);
    }
  }
  return out;
}

/* createLinearIndexList (grid.js:228-243): k outer, j, i inner; 1-based input */
static int32_t* index_list(int is, int ie, int js, int je, int ks, int ke, long d2, long d3, int* count) {
  const int ni = ie - is + 1, nj = je - js + 1, nk = ke - ks + 1;
  const int n = (ni > 0 && nj > 0 && nk > 0) ? ni * nj * nk : 0;
  int32_t* fi = (int32_t*)xcalloc(n, 4);
  int p = 0;
  for (int mk = ks; mk <= ke; mk++)
    for (int mj = js; mj <= je; mj++)
      for (int mi = is; mi <= ie; mi++) fi[p++] = (int32_t)((mi - 1) * d2 * d3 + (mj - 1) * d3 + (mk - 1));
  *count = n;
  return fi;
}

static void init_sources(ofd_state* g, const ofd_scn* s) {
  const double dx = g->dx, dy = g->dy, dz = g->dz, dt = g->dt;
  double maxCell = dx;
  if (dy > maxCell) maxCell = dy;
  if (dz > maxCell) maxCell = dz;
  g->n_wave = s->n_wave;
  g->waves = (double**)xcalloc(s->n_wave, sizeof(double*));
  for (int w = 0; w < s->n_wave; w++) g->waves[w] = make_waveform(s->wave + 4 * w, g->nsteps, dt, maxCell);

  g->n_vs = s->n_vs;
  g->vs = (ofd_vsrc*)xcalloc(s->n_vs, sizeof(ofd_vsrc));
  for (int n = 0; n < s->n_vs; n++) {
    const double* v = s->vs + 11 * n;
    ofd_vsrc* V = &g->vs[n];
    const int is = js_round((v[0] - g->min_x) / dx) + 1, js = js_round((v[1] - g->min_y) / dy) + 1,
              ks = js_round((v[2] - g->min_z) / dz) + 1;
    const int ie = js_round((v[3] - g->min_x) / dx) + 1, je = js_round((v[4] - g->min_y) / dy) + 1,
              ke = js_round((v[5] - g->min_z) / dz) + 1;
    const int axis = (int)v[6];
    const double sign = v[7];
    int n_fields;
    double r_factor;
    if (axis == 0) {
      n_fields = ie - is;
      r_factor = (double)((1 + je - js) * (1 + ke - ks)) / (ie - is);
    } else if (axis == 1) {
      n_fields = je - js;
      r_factor = (double)((1 + ie - is) * (1 + ke - ks)) / (je - js);
    } else {
      n_fields = ke - ks;
      r_factor = (double)((1 + ie - is) * (1 + je - js)) / (ke - ks);
    }
    const double v_mag = sign * v[9] / n_fields;
    V->resistance_per_component = r_factor * v[8];
    const double* base = g->waves[(int)v[10]];
    V->vpe = (double*)xcalloc(g->nsteps, 8);
    for (int t = 0; t < g->nsteps; t++) V->vpe[t] = v_mag * base[t];
    V->axis = axis;

    /* applyLumpedElementCoefficients, voltage-source branch (coefficients.js:158-207) */
    double R = V->resistance_per_component;
    if (R == 0) R = 1e-20;
    if (axis == 0) {
      V->fi = index_list(is, ie - 1, js, je, ks, ke, g->nyp1, g->nzp1, &V->n);
      const double a_term = (dt * dx) / (R * dy * dz);
      V->cs = (double*)xcalloc(V->n, 8);
      for (int q = 0; q < V->n; q++) {
        const long idx = V->fi[q];
        const double denom = 2 * EPS0 * g->eps_r_x[idx] + dt * g->sigma_e_x[idx] + a_term;
        g->Cexe[idx] = (2 * EPS0 * g->eps_r_x[idx] - dt * g->sigma_e_x[idx] - a_term) / denom;
        g->Cexhz[idx] = (2 * dt / dy) / denom;
        g->Cexhy[idx] = -(2 * dt / dz) / denom;
        V->cs[q] = -(2 * dt / (R * dy * dz)) / denom;
      }
    } else if (axis == 1) {
      V->fi = index_list(is, ie, js, je - 1, ks, ke, g->ny, g->nzp1, &V->n);
      const double a_term = (dt * dy) / (R * dz * dx);
      V->cs = (double*)xcalloc(V->n, 8);
      for (int q = 0; q < V->n; q++) {
        const long idx = V->fi[q];
        const double denom = 2 * EPS0 * g->eps_r_y[idx] + dt * g->sigma_e_y[idx] + a_term;
        g->Ceye[idx] = (2 * EPS0 * g->eps_r_y[idx] - dt * g->sigma_e_y[idx] - a_term) / denom;
        g->Ceyhx[idx] = (2 * dt / dz) / denom;
        g->Ceyhz[idx] = -(2 * dt / dx) / denom;
        V->cs[q] = -(2 * dt / (R * dz * dx)) / denom;
      }
    } else {
      V->fi = index_list(is, ie, js, je, ks, ke - 1, g->nyp1, g->nz, &V->n);
      const double a_term = (dt * dz) / (R * dx * dy);
      V->cs = (double*)xcalloc(V->n, 8);
      for (int q = 0; q < V->n; q++) {
        const long idx = V->fi[q];
        const double denom = 2 * EPS0 * g->eps_r_z[idx] + dt * g->sigma_e_z[idx] + a_term;
        g->Ceze[idx] = (2 * EPS0 * g->eps_r_z[idx] - dt * g->sigma_e_z[idx] - a_term) / denom;
        g->Cezhy[idx] = (2 * dt / dx) / denom;
        g->Cezhx[idx] = -(2 * dt / dy) / denom;
        V->cs[q] = -(2 * dt / (R * dx * dy)) / denom;
      }
    }
  }
}

/* sampling.js:81-136 */
static void init_samplers(ofd_state* g, const ofd_scn* s) {
  const double dx = g->dx, dy = g->dy, dz = g->dz;
  g->n_sv = s->n_sv;
  g->sv = (ofd_probe*)xcalloc(s->n_sv, sizeof(ofd_probe));
  for (int n = 0; n < s->n_sv; n++) {
    const double* v = s->sv + 8 * n;
    ofd_probe* P = &g->sv[n];
    P->is = js_round((v[0] - g->min_x) / dx) + 1; P->js = js_round((v[1] - g->min_y) / dy) + 1;
    P->ks = js_round((v[2] - g->min_z) / dz) + 1; P->ie = js_round((v[3] - g->min_x) / dx) + 1;
    P->je = js_round((v[4] - g->min_y) / dy) + 1; P->ke = js_round((v[5] - g->min_z) / dz) + 1;
    P->axis = (int)v[6]; P->sign = (int)v[7];
    if (P->axis == 0) {
      P->fi = index_list(P->is, P->ie - 1, P->js, P->je, P->ks, P->ke, g->nyp1, g->nzp1, &P->nfi);
      P->Csvf = -dx / ((P->je - P->js + 1) * (P->ke - P->ks + 1));
    } else if (P->axis == 1) {
      P->fi = index_list(P->is, P->ie, P->js, P->je - 1, P->ks, P->ke, g->ny, g->nzp1, &P->nfi);
      P->Csvf = -dy / ((P->ke - P->ks + 1) * (P->ie - P->is + 1));
    } else {
      P->fi = index_list(P->is, P->ie, P->js, P->je, P->ks, P->ke - 1, g->nyp1, g->nz, &P->nfi);
      P->Csvf = -dz / ((P->ie - P->is + 1) * (P->je - P->js + 1));
    }
    if (P->sign < 0) P->Csvf *= -1;
    P->val = (double*)xcalloc(g->nsteps, 8);
  }
  g->n_si = s->n_si;
  g->si = (ofd_probe*)xcalloc(s->n_si, sizeof(ofd_probe));
  for (int n = 0; n < s->n_si; n++) {
    const double* v = s->si + 8 * n;
    ofd_probe* P = &g->si[n];
    P->is = js_round((v[0] - g->min_x) / dx) + 1; P->js = js_round((v[1] - g->min_y) / dy) + 1;
    P->ks = js_round((v[2] - g->min_z) / dz) + 1; P->ie = js_round((v[3] - g->min_x) / dx) + 1;
    P->je = js_round((v[4] - g->min_y) / dy) + 1; P->ke = js_round((v[5] - g->min_z) / dz) + 1;
    P->axis = (int)v[6]; P->sign = (int)v[7];
    P->val = (double*)xcalloc(g->nsteps, 8);
  }
}

/* farfield.js:28-78 */
static void init_farfield(ofd_state* g, const ofd_scn* s) {
  g->nFreq = s->n_ff;
  if (g->nFreq == 0) return;
  const int nc = s->nc_ff;
  g->li = nc + 1; g->lj = nc + 1; g->lk = nc + 1;
  g->ui = g->nx - nc + 1; g->uj = g->ny - nc + 1; g->uk = g->nz - nc + 1;
  g->ni_ff = g->ui - g->li; g->nj_ff = g->uj - g->lj; g->nk_ff = g->uk - g->lk;
  g->sz_x = (long)g->nj_ff * g->nk_ff;
  g->sz_y = (long)g->ni_ff * g->nk_ff;
  g->sz_z = (long)g->ni_ff * g->nj_ff;
  g->ffreq = (double*)xcalloc(g->nFreq, 8);
  g->w = (double*)xcalloc(g->nFreq, 8);
  for (int m = 0; m < g->nFreq; m++) { g->ffreq[m] = s->ff_freq[m]; g->w[m] = 2 * M_PI * s->ff_freq[m]; }
  long tot = 0, sz[24];
  for (int a = 0; a < 24; a++) {
    const int fa = (a % 12) / 4; /* 0: x-face arrays, 1: y-face, 2: z-face */
    sz[a] = fa == 0 ? g->sz_x : (fa == 1 ? g->sz_y : g->sz_z);
    tot += 2 * sz[a] * g->nFreq;
  }
  g->ffacc = (double*)xcalloc(tot, 8);
  double* p = g->ffacc;
  for (int a = 0; a < 24; a++) {
    g->ffp[a][0] = p; p += sz[a] * g->nFreq;
    g->ffp[a][1] = p; p += sz[a] * g->nFreq;
  }
}

/* ------------------------------------------------------------------------- */
/* Per-step work                                                              */
/* ------------------------------------------------------------------------- */
/* fdtd_kernels.ts:20-114 */
static void update_h(ofd_state* g) {
  const long nx = g->nx, ny = g->ny, nz = g->nz, nxp1 = g->nxp1, nyp1 = g->nyp1, nzp1 = g->nzp1;
  double *Hx = g->Hx, *Hy = g->Hy, *Hz = g->Hz;
  const double *Ex = g->Ex, *Ey = g->Ey, *Ez = g->Ez;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < nxp1; i++)
    for (long j = 0; j < ny; j++) {
      const long hxOff = i * ny * nz + j * nz, eyOff = i * ny * nzp1 + j * nzp1;
      const long ezOff0 = i * nyp1 * nz + j * nz, ezOff1 = i * nyp1 * nz + (j + 1) * nz;
      for (long k = 0; k < nz; k++) {
        const long idx = hxOff + k;
        Hx[idx] = g->Chxh[idx] * Hx[idx] + g->Chxey[idx] * (Ey[eyOff + k + 1] - Ey[eyOff + k]) +
                  g->Chxez[idx] * (Ez[ezOff1 + k] - Ez[ezOff0 + k]);
      }
    }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < nx; i++)
    for (long j = 0; j < nyp1; j++) {
      const long hyOff = i * nyp1 * nz + j * nz;
      const long ezOff0 = i * nyp1 * nz + j * nz, ezOff1 = (i + 1) * nyp1 * nz + j * nz;
      const long exOff = i * nyp1 * nzp1 + j * nzp1;
      for (long k = 0; k < nz; k++) {
        const long idx = hyOff + k;
        Hy[idx] = g->Chyh[idx] * Hy[idx] + g->Chyez[idx] * (Ez[ezOff1 + k] - Ez[ezOff0 + k]) +
                  g->Chyex[idx] * (Ex[exOff + k + 1] - Ex[exOff + k]);
      }
    }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < nx; i++)
    for (long j = 0; j < ny; j++) {
      const long hzOff = i * ny * nzp1 + j * nzp1;
      const long exOff0 = i * nyp1 * nzp1 + j * nzp1, exOff1 = i * nyp1 * nzp1 + (j + 1) * nzp1;
      const long eyOff0 = i * ny * nzp1 + j * nzp1, eyOff1 = (i + 1) * ny * nzp1 + j * nzp1;
      for (long k = 0; k < nzp1; k++) {
        const long idx = hzOff + k;
        Hz[idx] = g->Chzh[idx] * Hz[idx] + g->Chzex[idx] * (Ex[exOff1 + k] - Ex[exOff0 + k]) +
                  g->Chzey[idx] * (Ey[eyOff1 + k] - Ey[eyOff0 + k]);
      }
    }
}

/* fdtd_kernels.ts:116-210.  Ey/Ez run i = 1..nx inclusive (partition end nxp1); at
 * i = nx the Hz[i]/Hy[i] reads fall one plane past those arrays, into the next
 * array of the contiguous field block, as in the reference's shared memory. */
static int g_edge_read_old = 0;
void ofd_set_edge_read(int old) { g_edge_read_old = old; }

static void update_e(ofd_state* g) {
  const long nx = g->nx, ny = g->ny, nz = g->nz, nxp1 = g->nxp1, nyp1 = g->nyp1, nzp1 = g->nzp1;
  const double *Hx = g->Hx, *Hy = g->Hy, *Hz = g->Hz;
  double *Ex = g->Ex, *Ey = g->Ey, *Ez = g->Ez;
  /* Hz one plane past its end is Ex(i=0,...): optionally freeze its pre-update copy */
  double* ex0_old = NULL;
  if (g_edge_read_old) {
    ex0_old = (double*)xcalloc((size_t)nyp1 * nzp1, 8);
    memcpy(ex0_old, Ex, sizeof(double) * nyp1 * nzp1);
  }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < nx; i++)
    for (long j = 1; j < ny; j++) {
      const long exOff = i * nyp1 * nzp1 + j * nzp1;
      const long hzOff0 = i * ny * nzp1 + (j - 1) * nzp1, hzOff1 = i * ny * nzp1 + j * nzp1;
      const long hyOff = i * nyp1 * nz + j * nz;
      for (long k = 1; k < nz; k++) {
        const long idx = exOff + k;
        Ex[idx] = g->Cexe[idx] * Ex[idx] + g->Cexhz[idx] * (Hz[hzOff1 + k] - Hz[hzOff0 + k]) +
                  g->Cexhy[idx] * (Hy[hyOff + k] - Hy[hyOff + k - 1]);
      }
    }
#pragma omp parallel for schedule(static)
  for (long i = 1; i < nxp1; i++)
    for (long j = 0; j < ny; j++) {
      const long eyOff = i * ny * nzp1 + j * nzp1, hxOff = i * ny * nz + j * nz;
      const long hzOff0 = (i - 1) * ny * nzp1 + j * nzp1, hzOff1 = i * ny * nzp1 + j * nzp1;
      for (long k = 1; k < nz; k++) {
        const long idx = eyOff + k;
        const double hz1 = (ex0_old && i == nx) ? ex0_old[hzOff1 + k - nx * ny * nzp1] : Hz[hzOff1 + k];
        Ey[idx] = g->Ceye[idx] * Ey[idx] + g->Ceyhx[idx] * (Hx[hxOff + k] - Hx[hxOff + k - 1]) +
                  g->Ceyhz[idx] * (hz1 - Hz[hzOff0 + k]);
      }
    }
  free(ex0_old);
#pragma omp parallel for schedule(static)
  for (long i = 1; i < nxp1; i++)
    for (long j = 1; j < ny; j++) {
      const long ezOff = i * nyp1 * nz + j * nz;
      const long hyOff0 = (i - 1) * nyp1 * nz + j * nz, hyOff1 = i * nyp1 * nz + j * nz;
      const long hxOff0 = i * ny * nz + (j - 1) * nz, hxOff1 = i * ny * nz + j * nz;
      for (long k = 0; k < nz; k++) {
        const long idx = ezOff + k;
        Ez[idx] = g->Ceze[idx] * Ez[idx] + g->Cezhy[idx] * (Hy[hyOff1 + k] - Hy[hyOff0 + k]) +
                  g->Cezhx[idx] * (Hx[hxOff1 + k] - Hx[hxOff0 + k]);
      }
    }
}

/* cpml.js:456-724.  Psi updates read only E; corrections only write H, applied
 * face by face in the reference's face order, so every H element receives its
 * corrections in the same sequence. */
static void update_mag_cpml(ofd_state* g) {
  const long nx = g->nx, ny = g->ny, nz = g->nz, nxp1 = g->nxp1, nyp1 = g->nyp1, nzp1 = g->nzp1;
  double *Hx = g->Hx, *Hy = g->Hy, *Hz = g->Hz;
  const double *Ex = g->Ex, *Ey = g->Ey, *Ez = g->Ez;
  for (int fid = 0; fid < 6; fid++) {
    if (!g->has_face[fid]) continue;
    ofd_face* f = &g->face[fid];
    const long nc = f->nc;
    double *P0 = f->psi[0], *P1 = f->psi[1], *C0p = f->cpsi[0], *C1p = f->cpsi[1];
    const long st = f->m_start;
    if (f->axis == 0) {
#pragma omp parallel for schedule(static)
      for (long ci = 0; ci < nc; ci++) {
        const double bm = f->b_m[ci], am = f->a_m[ci];
        const long ei = st + ci;
        for (long j = 0; j < nyp1; j++)
          for (long k = 0; k < nz; k++) {
            const long pi = ci * nyp1 * nz + j * nz + k;
            P0[pi] = bm * P0[pi] + am * (Ez[(ei + 1) * nyp1 * nz + j * nz + k] - Ez[ei * nyp1 * nz + j * nz + k]);
          }
        for (long j = 0; j < ny; j++)
          for (long k = 0; k < nzp1; k++) {
            const long pi = ci * ny * nzp1 + j * nzp1 + k;
            P1[pi] = bm * P1[pi] + am * (Ey[(ei + 1) * ny * nzp1 + j * nzp1 + k] - Ey[ei * ny * nzp1 + j * nzp1 + k]);
          }
      }
#pragma omp parallel for schedule(static)
      for (long ci = 0; ci < nc; ci++) {
        const long i = st + ci;
        for (long j = 0; j < nyp1; j++)
          for (long k = 0; k < nz; k++)
            Hy[i * nyp1 * nz + j * nz + k] += C0p[ci * nyp1 * nz + j * nz + k] * P0[ci * nyp1 * nz + j * nz + k];
        for (long j = 0; j < ny; j++)
          for (long k = 0; k < nzp1; k++)
            Hz[i * ny * nzp1 + j * nzp1 + k] += C1p[ci * ny * nzp1 + j * nzp1 + k] * P1[ci * ny * nzp1 + j * nzp1 + k];
      }
    } else if (f->axis == 1) {
      /* slot 0 = hxy (driven by Ez), slot 1 = hzy (driven by Ex) */
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nxp1; i++)
        for (long ci = 0; ci < nc; ci++) {
          const double bm = f->b_m[ci], am = f->a_m[ci];
          const long jh = st + ci;
          for (long k = 0; k < nz; k++) {
            const long pi = i * nc * nz + ci * nz + k;
            P0[pi] = bm * P0[pi] + am * (Ez[i * nyp1 * nz + (jh + 1) * nz + k] - Ez[i * nyp1 * nz + jh * nz + k]);
          }
        }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nx; i++)
        for (long ci = 0; ci < nc; ci++) {
          const double bm = f->b_m[ci], am = f->a_m[ci];
          const long jh = st + ci;
          for (long k = 0; k < nzp1; k++) {
            const long pi = i * nc * nzp1 + ci * nzp1 + k;
            P1[pi] = bm * P1[pi] + am * (Ex[i * nyp1 * nzp1 + (jh + 1) * nzp1 + k] - Ex[i * nyp1 * nzp1 + jh * nzp1 + k]);
          }
        }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nx; i++)
        for (long ci = 0; ci < nc; ci++) {
          const long j = st + ci;
          for (long k = 0; k < nzp1; k++)
            Hz[i * ny * nzp1 + j * nzp1 + k] += C1p[i * nc * nzp1 + ci * nzp1 + k] * P1[i * nc * nzp1 + ci * nzp1 + k];
        }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nxp1; i++)
        for (long ci = 0; ci < nc; ci++) {
          const long j = st + ci;
          for (long k = 0; k < nz; k++)
            Hx[i * ny * nz + j * nz + k] += C0p[i * nc * nz + ci * nz + k] * P0[i * nc * nz + ci * nz + k];
        }
    } else {
      /* slot 0 = hxz (driven by Ey), slot 1 = hyz (driven by Ex) */
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nxp1; i++)
        for (long j = 0; j < ny; j++)
          for (long ci = 0; ci < nc; ci++) {
            const long kh = st + ci, pi = i * ny * nc + j * nc + ci;
            P0[pi] = f->b_m[ci] * P0[pi] + f->a_m[ci] * (Ey[i * ny * nzp1 + j * nzp1 + (kh + 1)] - Ey[i * ny * nzp1 + j * nzp1 + kh]);
          }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nx; i++)
        for (long j = 0; j < nyp1; j++)
          for (long ci = 0; ci < nc; ci++) {
            const long kh = st + ci, pi = i * nyp1 * nc + j * nc + ci;
            P1[pi] = f->b_m[ci] * P1[pi] + f->a_m[ci] * (Ex[i * nyp1 * nzp1 + j * nzp1 + (kh + 1)] - Ex[i * nyp1 * nzp1 + j * nzp1 + kh]);
          }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nxp1; i++)
        for (long j = 0; j < ny; j++)
          for (long ci = 0; ci < nc; ci++) {
            const long k = st + ci, pi = i * ny * nc + j * nc + ci;
            Hx[i * ny * nz + j * nz + k] += C0p[pi] * P0[pi];
          }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nx; i++)
        for (long j = 0; j < nyp1; j++)
          for (long ci = 0; ci < nc; ci++) {
            const long k = st + ci, pi = i * nyp1 * nc + j * nc + ci;
            Hy[i * nyp1 * nz + j * nz + k] += C1p[pi] * P1[pi];
          }
    }
  }
}

/* cpml.js:727-1003 */
static void update_ele_cpml(ofd_state* g) {
  const long nx = g->nx, ny = g->ny, nz = g->nz, nxp1 = g->nxp1, nyp1 = g->nyp1, nzp1 = g->nzp1;
  const double *Hx = g->Hx, *Hy = g->Hy, *Hz = g->Hz;
  double *Ex = g->Ex, *Ey = g->Ey, *Ez = g->Ez;
  for (int fid = 0; fid < 6; fid++) {
    if (!g->has_face[fid]) continue;
    ofd_face* f = &g->face[fid];
    const long nc = f->nc;
    double *P2 = f->psi[2], *P3 = f->psi[3], *C2p = f->cpsi[2], *C3p = f->cpsi[3];
    const long st = f->e_start;
    /* source index of the lower H plane: xn uses ci, xp uses n_st + ci - 1 */
    const long src0 = f->ascending ? st - 1 : 0;
    if (f->axis == 0) {
      /* slot 2 = eyx (driven by Hz), slot 3 = ezx (driven by Hy) */
#pragma omp parallel for schedule(static)
      for (long ci = 0; ci < nc; ci++) {
        const double be = f->b_e[ci], ae = f->a_e[ci];
        const long hi = src0 + ci;
        for (long j = 0; j < ny; j++)
          for (long k = 0; k < nzp1; k++) {
            const long pi = ci * ny * nzp1 + j * nzp1 + k;
            P2[pi] = be * P2[pi] + ae * (Hz[(hi + 1) * ny * nzp1 + j * nzp1 + k] - Hz[hi * ny * nzp1 + j * nzp1 + k]);
          }
        for (long j = 0; j < nyp1; j++)
          for (long k = 0; k < nz; k++) {
            const long pi = ci * nyp1 * nz + j * nz + k;
            P3[pi] = be * P3[pi] + ae * (Hy[(hi + 1) * nyp1 * nz + j * nz + k] - Hy[hi * nyp1 * nz + j * nz + k]);
          }
      }
#pragma omp parallel for schedule(static)
      for (long ci = 0; ci < nc; ci++) {
        const long i = st + ci;
        for (long j = 0; j < ny; j++)
          for (long k = 0; k < nzp1; k++)
            Ey[i * ny * nzp1 + j * nzp1 + k] += C2p[ci * ny * nzp1 + j * nzp1 + k] * P2[ci * ny * nzp1 + j * nzp1 + k];
        for (long j = 0; j < nyp1; j++)
          for (long k = 0; k < nz; k++)
            Ez[i * nyp1 * nz + j * nz + k] += C3p[ci * nyp1 * nz + j * nz + k] * P3[ci * nyp1 * nz + j * nz + k];
      }
    } else if (f->axis == 1) {
      /* slot 2 = ezy (driven by Hx), slot 3 = exy (driven by Hz) */
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nxp1; i++)
        for (long ci = 0; ci < nc; ci++) {
          const double be = f->b_e[ci], ae = f->a_e[ci];
          const long hj = src0 + ci;
          for (long k = 0; k < nz; k++) {
            const long pi = i * nc * nz + ci * nz + k;
            P2[pi] = be * P2[pi] + ae * (Hx[i * ny * nz + (hj + 1) * nz + k] - Hx[i * ny * nz + hj * nz + k]);
          }
        }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nx; i++)
        for (long ci = 0; ci < nc; ci++) {
          const double be = f->b_e[ci], ae = f->a_e[ci];
          const long hj = src0 + ci;
          for (long k = 0; k < nzp1; k++) {
            const long pi = i * nc * nzp1 + ci * nzp1 + k;
            P3[pi] = be * P3[pi] + ae * (Hz[i * ny * nzp1 + (hj + 1) * nzp1 + k] - Hz[i * ny * nzp1 + hj * nzp1 + k]);
          }
        }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nxp1; i++)
        for (long ci = 0; ci < nc; ci++) {
          const long j = st + ci;
          for (long k = 0; k < nz; k++)
            Ez[i * nyp1 * nz + j * nz + k] += C2p[i * nc * nz + ci * nz + k] * P2[i * nc * nz + ci * nz + k];
        }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nx; i++)
        for (long ci = 0; ci < nc; ci++) {
          const long j = st + ci;
          for (long k = 0; k < nzp1; k++)
            Ex[i * nyp1 * nzp1 + j * nzp1 + k] += C3p[i * nc * nzp1 + ci * nzp1 + k] * P3[i * nc * nzp1 + ci * nzp1 + k];
        }
    } else {
      /* slot 2 = exz (driven by Hy), slot 3 = eyz (driven by Hx) */
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nx; i++)
        for (long j = 0; j < nyp1; j++)
          for (long ci = 0; ci < nc; ci++) {
            const long hk = src0 + ci, pi = i * nyp1 * nc + j * nc + ci;
            P2[pi] = f->b_e[ci] * P2[pi] + f->a_e[ci] * (Hy[i * nyp1 * nz + j * nz + (hk + 1)] - Hy[i * nyp1 * nz + j * nz + hk]);
          }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nxp1; i++)
        for (long j = 0; j < ny; j++)
          for (long ci = 0; ci < nc; ci++) {
            const long hk = src0 + ci, pi = i * ny * nc + j * nc + ci;
            P3[pi] = f->b_e[ci] * P3[pi] + f->a_e[ci] * (Hx[i * ny * nz + j * nz + (hk + 1)] - Hx[i * ny * nz + j * nz + hk]);
          }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nx; i++)
        for (long j = 0; j < nyp1; j++)
          for (long ci = 0; ci < nc; ci++) {
            const long k = st + ci, pi = i * nyp1 * nc + j * nc + ci;
            Ex[i * nyp1 * nzp1 + j * nzp1 + k] += C2p[pi] * P2[pi];
          }
#pragma omp parallel for schedule(static)
      for (long i = 0; i < nxp1; i++)
        for (long j = 0; j < ny; j++)
          for (long ci = 0; ci < nc; ci++) {
            const long k = st + ci, pi = i * ny * nc + j * nc + ci;
            Ey[i * ny * nzp1 + j * nzp1 + k] += C3p[pi] * P3[pi];
          }
    }
  }
}

/* sampling.js:204-245 */
static void capture_currents(ofd_state* g, int ts) {
  const long ny = g->ny, nz = g->nz, nyp1 = g->nyp1, nzp1 = g->nzp1;
  const double dx = g->dx, dy = g->dy, dz = g->dz;
#define IHX(i, j, k) ((long)(i) * ny * nz + (long)(j) * nz + (k))
#define IHY(i, j, k) ((long)(i) * nyp1 * nz + (long)(j) * nz + (k))
#define IHZ(i, j, k) ((long)(i) * ny * nzp1 + (long)(j) * nzp1 + (k))
  for (int n = 0; n < g->n_si; n++) {
    ofd_probe* P = &g->si[n];
    const int I = P->is - 1, J = P->js - 1, K = P->ks - 1, IE = P->ie - 1, JE = P->je - 1, KE = P->ke - 1;
    double sv = 0;
    if (P->axis == 0) {
      const int ix = IE - 1;
      for (int j = J; j <= JE - 1; j++) sv += dy * g->Hy[IHY(ix, j, K - 1)];
      for (int k = K; k <= KE - 1; k++) sv += dz * g->Hz[IHZ(ix, JE - 1, k)];
      for (int j = J; j <= JE - 1; j++) sv -= dy * g->Hy[IHY(ix, j, KE - 1)];
      for (int k = K; k <= KE - 1; k++) sv -= dz * g->Hz[IHZ(ix, J - 1, k)];
    } else if (P->axis == 1) {
      const int jx = JE - 1;
      for (int k = K; k <= KE - 1; k++) sv += dz * g->Hz[IHZ(I - 1, jx, k)];
      for (int i = I; i <= IE - 1; i++) sv += dx * g->Hx[IHX(i, jx, KE - 1)];
      for (int k = K; k <= KE - 1; k++) sv -= dz * g->Hz[IHZ(IE, jx, k)];
      for (int i = I; i <= IE - 1; i++) sv -= dx * g->Hx[IHX(i, jx, K - 1)];
    } else {
      const int kx = KE - 1;
      for (int i = I; i <= IE - 1; i++) sv += dx * g->Hx[IHX(i, J - 1, kx)];
      for (int j = J; j <= JE - 1; j++) sv += dy * g->Hy[IHY(IE, j, kx)];
      for (int i = I; i <= IE - 1; i++) sv -= dx * g->Hx[IHX(i, JE, kx)];
      for (int j = J; j <= JE - 1; j++) sv -= dy * g->Hy[IHY(I - 1, j, kx)];
    }
    if (P->sign < 0) sv = -sv;
    P->val[ts] = sv;
  }
}

/* sources.js:271-288 */
static void inject_sources(ofd_state* g, int ts) {
  for (int n = 0; n < g->n_vs; n++) {
    ofd_vsrc* V = &g->vs[n];
    const double v = V->vpe[ts];
    double* F = V->axis == 0 ? g->Ex : (V->axis == 1 ? g->Ey : g->Ez);
    for (int q = 0; q < V->n; q++) F[V->fi[q]] += V->cs[q] * v;
  }
}

/* sampling.js:295-307 */
static void capture_voltages(ofd_state* g, int ts) {
  for (int n = 0; n < g->n_sv; n++) {
    ofd_probe* P = &g->sv[n];
    const double* F = P->axis == 0 ? g->Ex : (P->axis == 1 ? g->Ey : g->Ez);
    double sum = 0;
    for (int q = 0; q < P->nfi; q++) sum += F[P->fi[q]];
    P->val[ts] = P->Csvf * sum;
  }
}

/* farfield.js:90-248 */
static void accumulate_ff(ofd_state* g, int ts) {
  if (g->nFreq == 0) return;
  const long ny = g->ny, nz = g->nz, nyp1 = g->nyp1, nzp1 = g->nzp1;
  const double *Hx = g->Hx, *Hy = g->Hy, *Hz = g->Hz, *Ex = g->Ex, *Ey = g->Ey, *Ez = g->Ez;
  const int LI = g->li - 1, LJ = g->lj - 1, LK = g->lk - 1, UI = g->ui - 1, UJ = g->uj - 1, UK = g->uk - 1;
  const int ni_ff = g->ni_ff, nj_ff = g->nj_ff, nk_ff = g->nk_ff;
#define IEX(i, j, k) ((long)(i) * nyp1 * nzp1 + (long)(j) * nzp1 + (k))
#define IEY(i, j, k) ((long)(i) * ny * nzp1 + (long)(j) * nzp1 + (k))
#define IEZ(i, j, k) ((long)(i) * nyp1 * nz + (long)(j) * nz + (k))
#define ACC(a, p, cr, ci, t) do { g->ffp[a][0][p] += (cr) * (t); g->ffp[a][1][p] += (ci) * (t); } while (0)
  for (int mi = 0; mi < g->nFreq; mi++) {
    const double wdt = g->w[mi] * g->dt;
    const double ph_h = wdt * (ts + 0.5);
    const double cos_h = cos(ph_h), sin_h = -sin(ph_h);
    const double ph_e = wdt * (ts + 1);
    const double cos_e = cos(ph_e), sin_e = -sin(ph_e);
    const long fx = mi * g->sz_x, fy = mi * g->sz_y, fz = mi * g->sz_z;
#pragma omp parallel for schedule(static)
    for (int nj = 0; nj < nj_ff; nj++)
      for (int nk = 0; nk < nk_ff; nk++) {
        const long p = fx + (long)nj * nk_ff + nk;
        const int j0 = LJ + nj, k0 = LK + nk;
        const double tmyxp = 0.5 * (Ez[IEZ(UI, j0, k0)] + Ez[IEZ(UI, j0 + 1, k0)]);
        ACC(CMYXP, p, cos_e, sin_e, tmyxp);
        const double tmzxp = -0.5 * (Ey[IEY(UI, j0, k0)] + Ey[IEY(UI, j0, k0 + 1)]);
        ACC(CMZXP, p, cos_e, sin_e, tmzxp);
        const double tjyxp = -0.25 * (Hz[IHZ(UI, j0, k0)] + Hz[IHZ(UI, j0, k0 + 1)] + Hz[IHZ(UI - 1, j0, k0)] + Hz[IHZ(UI - 1, j0, k0 + 1)]);
        ACC(CJYXP, p, cos_h, sin_h, tjyxp);
        const double tjzxp = 0.25 * (Hy[IHY(UI, j0, k0)] + Hy[IHY(UI, j0 + 1, k0)] + Hy[IHY(UI - 1, j0, k0)] + Hy[IHY(UI - 1, j0 + 1, k0)]);
        ACC(CJZXP, p, cos_h, sin_h, tjzxp);
        const double tmyxn = -0.5 * (Ez[IEZ(LI, j0, k0)] + Ez[IEZ(LI, j0 + 1, k0)]);
        ACC(CMYXN, p, cos_e, sin_e, tmyxn);
        const double tmzxn = 0.5 * (Ey[IEY(LI, j0, k0)] + Ey[IEY(LI, j0, k0 + 1)]);
        ACC(CMZXN, p, cos_e, sin_e, tmzxn);
        const double tjyxn = 0.25 * (Hz[IHZ(LI, j0, k0)] + Hz[IHZ(LI, j0, k0 + 1)] + Hz[IHZ(LI - 1, j0, k0)] + Hz[IHZ(LI - 1, j0, k0 + 1)]);
        ACC(CJYXN, p, cos_h, sin_h, tjyxn);
        const double tjzxn = -0.25 * (Hy[IHY(LI, j0, k0)] + Hy[IHY(LI, j0 + 1, k0)] + Hy[IHY(LI - 1, j0, k0)] + Hy[IHY(LI - 1, j0 + 1, k0)]);
        ACC(CJZXN, p, cos_h, sin_h, tjzxn);
      }
#pragma omp parallel for schedule(static)
    for (int ni = 0; ni < ni_ff; ni++)
      for (int nk = 0; nk < nk_ff; nk++) {
        const long p = fy + (long)ni * nk_ff + nk;
        const int i0 = LI + ni, k0 = LK + nk;
        const double tmxyp = -0.5 * (Ez[IEZ(i0, UJ, k0)] + Ez[IEZ(i0 + 1, UJ, k0)]);
        ACC(CMXYP, p, cos_e, sin_e, tmxyp);
        const double tmzyp = 0.5 * (Ex[IEX(i0, UJ, k0)] + Ex[IEX(i0, UJ, k0 + 1)]);
        ACC(CMZYP, p, cos_e, sin_e, tmzyp);
        const double tjzyp = -0.25 * (Hx[IHX(i0, UJ, k0)] + Hx[IHX(i0 + 1, UJ, k0)] + Hx[IHX(i0, UJ - 1, k0)] + Hx[IHX(i0 + 1, UJ - 1, k0)]);
        ACC(CJZYP, p, cos_h, sin_h, tjzyp);
        const double tjxyp = 0.25 * (Hz[IHZ(i0, UJ, k0)] + Hz[IHZ(i0, UJ, k0 + 1)] + Hz[IHZ(i0, UJ - 1, k0)] + Hz[IHZ(i0, UJ - 1, k0 + 1)]);
        ACC(CJXYP, p, cos_h, sin_h, tjxyp);
        const double tmxyn = 0.5 * (Ez[IEZ(i0, LJ, k0)] + Ez[IEZ(i0 + 1, LJ, k0)]);
        ACC(CMXYN, p, cos_e, sin_e, tmxyn);
        const double tmzyn = -0.5 * (Ex[IEX(i0, LJ, k0)] + Ex[IEX(i0, LJ, k0 + 1)]);
        ACC(CMZYN, p, cos_e, sin_e, tmzyn);
        const double tjzyn = 0.25 * (Hx[IHX(i0, LJ, k0)] + Hx[IHX(i0 + 1, LJ, k0)] + Hx[IHX(i0, LJ - 1, k0)] + Hx[IHX(i0 + 1, LJ - 1, k0)]);
        ACC(CJZYN, p, cos_h, sin_h, tjzyn);
        const double tjxyn = -0.25 * (Hz[IHZ(i0, LJ, k0)] + Hz[IHZ(i0, LJ, k0 + 1)] + Hz[IHZ(i0, LJ - 1, k0)] + Hz[IHZ(i0, LJ - 1, k0 + 1)]);
        ACC(CJXYN, p, cos_h, sin_h, tjxyn);
      }
#pragma omp parallel for schedule(static)
    for (int ni = 0; ni < ni_ff; ni++)
      for (int nj = 0; nj < nj_ff; nj++) {
        const long p = fz + (long)ni * nj_ff + nj;
        const int i0 = LI + ni, j0 = LJ + nj;
        const double tmxzp = 0.5 * (Ey[IEY(i0, j0, UK)] + Ey[IEY(i0 + 1, j0, UK)]);
        ACC(CMXZP, p, cos_e, sin_e, tmxzp);
        const double tmyzp = -0.5 * (Ex[IEX(i0, j0, UK)] + Ex[IEX(i0, j0 + 1, UK)]);
        ACC(CMYZP, p, cos_e, sin_e, tmyzp);
        const double tjxzp = 0.25 * (Hx[IHX(i0, j0, UK)] + Hx[IHX(i0 + 1, j0, UK)] + Hx[IHX(i0, j0, UK - 1)] + Hx[IHX(i0 + 1, j0, UK - 1)]);
        ACC(CJXZP, p, cos_h, sin_h, tjxzp);
        const double tjyzp2 = 0.25 * (Hx[IHX(i0, j0, UK)] + Hx[IHX(i0 + 1, j0, UK)] + Hx[IHX(i0, j0, UK - 1)] + Hx[IHX(i0 + 1, j0, UK - 1)]);
        const double tjxzp2 = -0.25 * (Hy[IHY(i0, j0, UK)] + Hy[IHY(i0, j0 + 1, UK)] + Hy[IHY(i0, j0, UK - 1)] + Hy[IHY(i0, j0 + 1, UK - 1)]);
        g->ffp[CJXZP][0][p] = g->ffp[CJXZP][0][p] - cos_h * tjxzp + cos_h * tjxzp2;
        g->ffp[CJXZP][1][p] = g->ffp[CJXZP][1][p] - sin_h * tjxzp + sin_h * tjxzp2;
        ACC(CJYZP, p, cos_h, sin_h, tjyzp2);
        const double tmxzn = -0.5 * (Ey[IEY(i0, j0, LK)] + Ey[IEY(i0 + 1, j0, LK)]);
        ACC(CMXZN, p, cos_e, sin_e, tmxzn);
        const double tmyzn = 0.5 * (Ex[IEX(i0, j0, LK)] + Ex[IEX(i0, j0 + 1, LK)]);
        ACC(CMYZN, p, cos_e, sin_e, tmyzn);
        const double tjxzn = 0.25 * (Hy[IHY(i0, j0, LK)] + Hy[IHY(i0, j0 + 1, LK)] + Hy[IHY(i0, j0, LK - 1)] + Hy[IHY(i0, j0 + 1, LK - 1)]);
        ACC(CJXZN, p, cos_h, sin_h, tjxzn);
        const double tjyzn = -0.25 * (Hx[IHX(i0, j0, LK)] + Hx[IHX(i0 + 1, j0, LK)] + Hx[IHX(i0, j0, LK - 1)] + Hx[IHX(i0 + 1, j0, LK - 1)]);
        ACC(CJYZN, p, cos_h, sin_h, tjyzn);
      }
  }
#undef ACC
}

/* ------------------------------------------------------------------------- */
/* Public entry points (ctypes)                                               */
/* ------------------------------------------------------------------------- */
void* ofd_create(const ofd_scn* s) {
  ofd_state* g = (ofd_state*)xcalloc(1, sizeof(ofd_state));
  g->nsteps = s->nsteps;
  build_grid(g, s);
  build_materials(g, s);
  general_coefficients(g);
  for (int f = 0; f < 6; f++) {
    g->has_face[f] = s->is_cpml[f];
    if (s->is_cpml[f]) init_face(g, s, f);
  }
  init_sources(g, s);
  init_samplers(g, s);
  init_farfield(g, s);
  return g;
}

void ofd_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int ofd_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Runs `count` steps from the current step; returns the new step index. */
int ofd_step(void* h, int count) {
  ofd_state* g = (ofd_state*)h;
  for (int c = 0; c < count && g->ts < g->nsteps; c++) {
    const int ts = g->ts;
    update_h(g);
    update_mag_cpml(g);
    capture_currents(g, ts);
    update_e(g);
    update_ele_cpml(g);
    inject_sources(g, ts);
    capture_voltages(g, ts);
    accumulate_ff(g, ts);
    g->ts++;
  }
  return g->ts;
}

/* Scalar metadata: ints[0..]=nx,ny,nz,nsteps,ts,nFreq,li,lj,lk,ui,uj,uk,n_vs,n_sv,n_si
 *                  dbl[0..]=dx,dy,dz,dt,min_x,min_y,min_z,max_x,max_y,max_z */
void ofd_meta(void* h, int* ints, double* dbl) {
  ofd_state* g = (ofd_state*)h;
  int v[15] = {g->nx, g->ny, g->nz, g->nsteps, g->ts, g->nFreq, g->li, g->lj, g->lk, g->ui, g->uj, g->uk,
               g->n_vs, g->n_sv, g->n_si};
  memcpy(ints, v, sizeof(v));
  double d[10] = {g->dx, g->dy, g->dz, g->dt, g->min_x, g->min_y, g->min_z, g->max_x, g->max_y, g->max_z};
  memcpy(dbl, d, sizeof(d));
}

/* Named array access.  Names: Hx..Ez, the 18 coefficient names, eps_r_x.. ,
 * "psi:<face>:<slot>", "cpsi:<face>:<slot>", "b_e:<face>" (b_e a_e b_m a_m kappa_e kappa_m),
 * "V:<n>", "I:<n>", "vfi:<n>" (source gap indices), "vcs:<n>", "vpe:<n>",
 * "svfi:<n>", "ff:<name>:re|im", "mat".  Returns the element count, or -1 if unknown;
 * copies min(count, cap) doubles to out when out != NULL. */
static long get_ptr(ofd_state* g, const char* name, const double** pd, const int32_t** pi, const uint8_t** pu) {
  *pd = NULL; *pi = NULL; *pu = NULL;
  struct { const char* n; double* p; long c; } tab[] = {
      {"Hx", g->Hx, g->nhx}, {"Hy", g->Hy, g->nhy}, {"Hz", g->Hz, g->nhz},
      {"Ex", g->Ex, g->nex}, {"Ey", g->Ey, g->ney}, {"Ez", g->Ez, g->nez},
      {"Cexe", g->Cexe, g->nex}, {"Cexhz", g->Cexhz, g->nex}, {"Cexhy", g->Cexhy, g->nex},
      {"Ceye", g->Ceye, g->ney}, {"Ceyhx", g->Ceyhx, g->ney}, {"Ceyhz", g->Ceyhz, g->ney},
      {"Ceze", g->Ceze, g->nez}, {"Cezhy", g->Cezhy, g->nez}, {"Cezhx", g->Cezhx, g->nez},
      {"Chxh", g->Chxh, g->nhx}, {"Chxez", g->Chxez, g->nhx}, {"Chxey", g->Chxey, g->nhx},
      {"Chyh", g->Chyh, g->nhy}, {"Chyex", g->Chyex, g->nhy}, {"Chyez", g->Chyez, g->nhy},
      {"Chzh", g->Chzh, g->nhz}, {"Chzey", g->Chzey, g->nhz}, {"Chzex", g->Chzex, g->nhz},
      {"eps_r_x", g->eps_r_x, g->nex}, {"eps_r_y", g->eps_r_y, g->ney}, {"eps_r_z", g->eps_r_z, g->nez},
      {"sigma_e_x", g->sigma_e_x, g->nex}, {"sigma_e_y", g->sigma_e_y, g->ney}, {"sigma_e_z", g->sigma_e_z, g->nez},
      {"mu_r_x", g->mu_r_x, g->nhx}, {"mu_r_y", g->mu_r_y, g->nhy}, {"mu_r_z", g->mu_r_z, g->nhz},
      {"sigma_m_x", g->sigma_m_x, g->nhx}, {"sigma_m_y", g->sigma_m_y, g->nhy}, {"sigma_m_z", g->sigma_m_z, g->nhz},
  };
  for (size_t t = 0; t < sizeof(tab) / sizeof(tab[0]); t++)
    if (!strcmp(name, tab[t].n)) { *pd = tab[t].p; return tab[t].c; }
  if (!strcmp(name, "mat")) { *pu = g->mat; return (long)g->nx * g->ny * g->nz; }
  int a = -1, b = -1;
  char buf[32];
  if (sscanf(name, "psi:%d:%d", &a, &b) == 2 && a >= 0 && a < 6 && g->has_face[a] && b >= 0 && b < 4) {
    *pd = g->face[a].psi[b]; return g->face[a].npsi[b];
  }
  if (sscanf(name, "cpsi:%d:%d", &a, &b) == 2 && a >= 0 && a < 6 && g->has_face[a] && b >= 0 && b < 4) {
    *pd = g->face[a].cpsi[b]; return g->face[a].npsi[b];
  }
  if (sscanf(name, "prof:%d:%d", &a, &b) == 2 && a >= 0 && a < 6 && g->has_face[a] && b >= 0 && b < 6) {
    ofd_face* f = &g->face[a];
    double* arr[6] = {f->b_e, f->a_e, f->b_m, f->a_m, f->kappa_e, f->kappa_m};
    *pd = arr[b]; return f->nc;
  }
  if (sscanf(name, "V:%d", &a) == 1 && a >= 0 && a < g->n_sv) { *pd = g->sv[a].val; return g->nsteps; }
  if (sscanf(name, "I:%d", &a) == 1 && a >= 0 && a < g->n_si) { *pd = g->si[a].val; return g->nsteps; }
  if (sscanf(name, "vcs:%d", &a) == 1 && a >= 0 && a < g->n_vs) { *pd = g->vs[a].cs; return g->vs[a].n; }
  if (sscanf(name, "vpe:%d", &a) == 1 && a >= 0 && a < g->n_vs) { *pd = g->vs[a].vpe; return g->nsteps; }
  if (sscanf(name, "vfi:%d", &a) == 1 && a >= 0 && a < g->n_vs) { *pi = g->vs[a].fi; return g->vs[a].n; }
  if (sscanf(name, "svfi:%d", &a) == 1 && a >= 0 && a < g->n_sv) { *pi = g->sv[a].fi; return g->sv[a].nfi; }
  if (sscanf(name, "svcsvf:%d", &a) == 1 && a >= 0 && a < g->n_sv) { *pd = &g->sv[a].Csvf; return 1; }
  if (sscanf(name, "sibox:%d", &a) == 1 && a >= 0 && a < g->n_si) { *pi = &g->si[a].is; return 6; }
  if (sscanf(name, "ff:%31[^:]:%d", buf, &b) == 2 && g->nFreq > 0 && (b == 0 || b == 1)) {
    for (int q = 0; q < 24; q++)
      if (!strcmp(buf, FF_NAMES[q])) {
        const int fa = (q % 12) / 4;
        *pd = g->ffp[q][b];
        return (fa == 0 ? g->sz_x : (fa == 1 ? g->sz_y : g->sz_z)) * g->nFreq;
      }
  }
  return -1;
}

long ofd_get(void* h, const char* name, double* out, long cap) {
  const double* pd; const int32_t* pi; const uint8_t* pu;
  long n = get_ptr((ofd_state*)h, name, &pd, &pi, &pu);
  if (n < 0 || !out) return n;
  long m = n < cap ? n : cap;
  for (long q = 0; q < m; q++) out[q] = pd ? pd[q] : (pi ? (double)pi[q] : (double)pu[q]);
  return n;
}

/* Overwrite a named double array (used by tests to plant state or perturbations). */
long ofd_set(void* h, const char* name, const double* in, long n) {
  const double* pd; const int32_t* pi; const uint8_t* pu;
  long c = get_ptr((ofd_state*)h, name, &pd, &pi, &pu);
  if (c < 0 || !pd || n != c) return -1;
  memcpy((double*)pd, in, n * sizeof(double));
  return n;
}

void ofd_destroy(void* h) {
  ofd_state* g = (ofd_state*)h;
  if (!g) return;
  free(g->fields); free(g->coef); free(g->mat);
  free(g->eps_r_x); free(g->eps_r_y); free(g->eps_r_z); free(g->mu_r_x); free(g->mu_r_y); free(g->mu_r_z);
  free(g->sigma_e_x); free(g->sigma_e_y); free(g->sigma_e_z); free(g->sigma_m_x); free(g->sigma_m_y); free(g->sigma_m_z);
  for (int f = 0; f < 6; f++) {
    if (!g->has_face[f]) continue;
    ofd_face* F = &g->face[f];
    free(F->b_e); free(F->a_e); free(F->b_m); free(F->a_m); free(F->kappa_e); free(F->kappa_m);
    for (int q = 0; q < 4; q++) { free(F->psi[q]); free(F->cpsi[q]); }
  }
  for (int n = 0; n < g->n_vs; n++) { free(g->vs[n].fi); free(g->vs[n].cs); free(g->vs[n].vpe); }
  for (int n = 0; n < g->n_sv; n++) { free(g->sv[n].fi); free(g->sv[n].val); }
  for (int n = 0; n < g->n_si; n++) free(g->si[n].val);
  for (int w = 0; w < g->n_wave; w++) free(g->waves[w]);
  free(g->waves); free(g->vs); free(g->sv); free(g->si);
  free(g->ffreq); free(g->w); free(g->ffacc);
  free(g);
}

/* ------------------------------------------------------------------------- */
/* Post-processing                                                            */
/* ------------------------------------------------------------------------- */
/* dft.js:17-38 */
void ofd_time_to_freq(const double* x, int N, double dt, const double* f, int M, double shift, double* re, double* im) {
#pragma omp parallel for schedule(static)
  for (int mi = 0; mi < M; mi++) {
    const double w = 2 * M_PI * f[mi];
    double r = 0, q = 0;
    for (int n = 0; n < N; n++) {
      const double t = (n + 1) * dt + shift;
      const double phase = w * t;
      r += x[n] * cos(phase);
      q -= x[n] * sin(phase);
    }
    re[mi] = r * dt;
    im[mi] = q * dt;
  }
}

/* sparameters.js:118-196 for one port that is its own source (S11). */
void ofd_s11(const double* Vre, const double* Vim, const double* Ire, const double* Iim, int M, double Z,
             double* Sre, double* Sim, double* mag_dB, double* phase_deg) {
  const double sq = sqrt(Z);
  for (int fi = 0; fi < M; fi++) {
    const double aRe = 0.5 * (Vre[fi] + Z * Ire[fi]) / sq;
    const double aIm = 0.5 * (Vim[fi] + Z * Iim[fi]) / sq;
    const double bRe = 0.5 * (Vre[fi] - Z * Ire[fi]) / sq;
    const double bIm = 0.5 * (Vim[fi] - Z * Iim[fi]) / sq;
    const double denom = aRe * aRe + aIm * aIm;
    if (denom < 1e-300) { Sre[fi] = 0; Sim[fi] = 0; }
    else {
      Sre[fi] = (bRe * aRe + bIm * aIm) / denom;
      Sim[fi] = (bIm * aRe - bRe * aIm) / denom;
    }
    const double mag = sqrt(Sre[fi] * Sre[fi] + Sim[fi] * Sim[fi]);
    mag_dB[fi] = mag > 0 ? 20 * log10(mag) : -INFINITY;
    phase_deg[fi] = atan2(Sim[fi], Sre[fi]) * 180 / M_PI;
  }
}

/* farfield.js:257-314 */
void ofd_radiated_power(void* h, double* out) {
  ofd_state* g = (ofd_state*)h;
  const double dx = g->dx, dy = g->dy, dz = g->dz;
  double* const(*F)[2] = g->ffp;
  for (int mi = 0; mi < g->nFreq; mi++) {
    const long ox = mi * g->sz_x, oy = mi * g->sz_y, oz = mi * g->sz_z;
    double powr = 0;
#define R(a, p) F[a][0][p]
#define I(a, p) F[a][1][p]
    for (long p = 0; p < g->sz_z; p++)
      powr += dx * dy * (R(CMYZP, oz + p) * R(CJXZP, oz + p) + I(CMYZP, oz + p) * I(CJXZP, oz + p) -
                         R(CMXZP, oz + p) * R(CJYZP, oz + p) - I(CMXZP, oz + p) * I(CJYZP, oz + p));
    for (long p = 0; p < g->sz_z; p++)
      powr -= dx * dy * (R(CMYZN, oz + p) * R(CJXZN, oz + p) + I(CMYZN, oz + p) * I(CJXZN, oz + p) -
                         R(CMXZN, oz + p) * R(CJYZN, oz + p) - I(CMXZN, oz + p) * I(CJYZN, oz + p));
    for (long p = 0; p < g->sz_y; p++)
      powr += dx * dz * (R(CMXYP, oy + p) * R(CJZYP, oy + p) + I(CMXYP, oy + p) * I(CJZYP, oy + p) -
                         R(CMZYP, oy + p) * R(CJXYP, oy + p) - I(CMZYP, oy + p) * I(CJXYP, oy + p));
    for (long p = 0; p < g->sz_y; p++)
      powr -= dx * dz * (R(CMXYN, oy + p) * R(CJZYN, oy + p) + I(CMXYN, oy + p) * I(CJZYN, oy + p) -
                         R(CMZYN, oy + p) * R(CJXYN, oy + p) - I(CMZYN, oy + p) * I(CJXYN, oy + p));
    for (long p = 0; p < g->sz_x; p++)
      powr += dy * dz * (R(CMZXP, ox + p) * R(CJYXP, ox + p) + I(CMZXP, ox + p) * I(CJYXP, ox + p) -
                         R(CMYXP, ox + p) * R(CJZXP, ox + p) - I(CMYXP, ox + p) * I(CJZXP, ox + p));
    for (long p = 0; p < g->sz_x; p++)
      powr -= dy * dz * (R(CMZXN, ox + p) * R(CJYXN, ox + p) + I(CMZXN, ox + p) * I(CJYXN, ox + p) -
                         R(CMYXN, ox + p) * R(CJZXN, ox + p) - I(CMYXN, ox + p) * I(CJZXN, ox + p));
#undef R
#undef I
    out[mi] = 0.5 * powr;
  }
}

/* farfield.js:328-607.  Angles run in parallel; for each angle the surface
 * terms are summed in the reference's face/point order. */
void ofd_directivity(void* h, const double* radP, const double* theta, const double* phi, int nA,
                     double* dTheta, double* dPhi) {
  ofd_state* g = (ofd_state*)h;
  const double dx = g->dx, dy = g->dy, dz = g->dz;
  const int li = g->li, lj = g->lj, lk = g->lk, ui = g->ui, uj = g->uj, uk = g->uk;
  const int ni_ff = g->ni_ff, nj_ff = g->nj_ff, nk_ff = g->nk_ff;
  const double ci = 0.5 * (ui + li), cj = 0.5 * (uj + lj), ck = 0.5 * (uk + lk);
  double* const(*F)[2] = g->ffp;
  for (int mi = 0; mi < g->nFreq; mi++) {
    const double k_wave = 2 * M_PI * g->ffreq[mi] / C0;
    const double scale = k_wave * k_wave / (8 * M_PI * ETA0 * radP[mi]);
    const long ox = mi * g->sz_x, oy = mi * g->sz_y, oz = mi * g->sz_z;
#pragma omp parallel for schedule(dynamic, 4)
    for (int a = 0; a < nA; a++) {
      const double sinth = sin(theta[a]), costh = cos(theta[a]), sinph = sin(phi[a]), cosph = cos(phi[a]);
      double NtRe = 0, NtIm = 0, NpRe = 0, NpIm = 0, LtRe = 0, LtIm = 0, LpRe = 0, LpIm = 0;
#define ROT(TR, TI, c, s, AR, AI) do { AR += (TR) * (c) - (TI) * (s); AI += (TR) * (s) + (TI) * (c); } while (0)
      for (int nj = 0; nj < nj_ff; nj++)
        for (int nk = 0; nk < nk_ff; nk++) {
          const long p = ox + (long)nj * nk_ff + nk;
          const int jpos = (lj - 1) + nj, kpos = (lk - 1) + nk;
          const double Jyr = F[CJYXP][0][p], Jyi = F[CJYXP][1][p], Jzr = F[CJZXP][0][p], Jzi = F[CJZXP][1][p];
          const double Myr = F[CMYXP][0][p], Myi = F[CMYXP][1][p], Mzr = F[CMZXP][0][p], Mzi = F[CMZXP][1][p];
          const double JyrN = F[CJYXN][0][p], JyiN = F[CJYXN][1][p], JzrN = F[CJZXN][0][p], JziN = F[CJZXN][1][p];
          const double MyrN = F[CMYXN][0][p], MyiN = F[CMYXN][1][p], MzrN = F[CMZXN][0][p], MziN = F[CMZXN][1][p];
          const double dydz = dy * dz;
          const double rpr_p = (ui - ci) * dx * sinth * cosph + (jpos - cj + 0.5) * dy * sinth * sinph + (kpos - ck + 0.5) * dz * costh;
          const double cp = cos(k_wave * rpr_p), sp = sin(k_wave * rpr_p);
          const double costh_sinph = costh * sinph;
          const double dydz_costh_sinph = dydz * costh_sinph, dydz_sinth = dydz * sinth, dydz_cosph = dydz * cosph;
          ROT(Jyr * dydz_costh_sinph - Jzr * dydz_sinth, Jyi * dydz_costh_sinph - Jzi * dydz_sinth, cp, sp, NtRe, NtIm);
          ROT(Jyr * dydz_cosph, Jyi * dydz_cosph, cp, sp, NpRe, NpIm);
          ROT(Myr * dydz_costh_sinph - Mzr * dydz_sinth, Myi * dydz_costh_sinph - Mzi * dydz_sinth, cp, sp, LtRe, LtIm);
          ROT(Myr * dydz_cosph, Myi * dydz_cosph, cp, sp, LpRe, LpIm);
          const double rpr_n = (li - ci) * dx * sinth * cosph + (jpos - cj + 0.5) * dy * sinth * sinph + (kpos - ck + 0.5) * dz * costh;
          const double cn = cos(k_wave * rpr_n), sn = sin(k_wave * rpr_n);
          ROT(JyrN * dydz_costh_sinph - JzrN * dydz_sinth, JyiN * dydz_costh_sinph - JziN * dydz_sinth, cn, sn, NtRe, NtIm);
          ROT(JyrN * dydz_cosph, JyiN * dydz_cosph, cn, sn, NpRe, NpIm);
          ROT(MyrN * dydz_costh_sinph - MzrN * dydz_sinth, MyiN * dydz_costh_sinph - MziN * dydz_sinth, cn, sn, LtRe, LtIm);
          ROT(MyrN * dydz_cosph, MyiN * dydz_cosph, cn, sn, LpRe, LpIm);
        }
      for (int ni = 0; ni < ni_ff; ni++)
        for (int nk = 0; nk < nk_ff; nk++) {
          const long p = oy + (long)ni * nk_ff + nk;
          const int ipos = (li - 1) + ni, kpos = (lk - 1) + nk;
          const double Jxr = F[CJXYP][0][p], Jxi = F[CJXYP][1][p], Jzr = F[CJZYP][0][p], Jzi = F[CJZYP][1][p];
          const double Mxr = F[CMXYP][0][p], Mxi = F[CMXYP][1][p], Mzr = F[CMZYP][0][p], Mzi = F[CMZYP][1][p];
          const double JxrN = F[CJXYN][0][p], JxiN = F[CJXYN][1][p], JzrN = F[CJZYN][0][p], JziN = F[CJZYN][1][p];
          const double MxrN = F[CMXYN][0][p], MxiN = F[CMXYN][1][p], MzrN = F[CMZYN][0][p], MziN = F[CMZYN][1][p];
          const double dxdz = dx * dz;
          const double rpr_p = (ipos - ci + 0.5) * dx * sinth * cosph + (uj - cj) * dy * sinth * sinph + (kpos - ck + 0.5) * dz * costh;
          const double cp = cos(k_wave * rpr_p), sp = sin(k_wave * rpr_p);
          const double costh_cosph = costh * cosph;
          const double dxdz_costh_cosph = dxdz * costh_cosph, dxdz_sinth = dxdz * sinth, dxdz_sinph = dxdz * sinph;
          ROT(Jxr * dxdz_costh_cosph - Jzr * dxdz_sinth, Jxi * dxdz_costh_cosph - Jzi * dxdz_sinth, cp, sp, NtRe, NtIm);
          ROT(-Jxr * dxdz_sinph, -Jxi * dxdz_sinph, cp, sp, NpRe, NpIm);
          ROT(Mxr * dxdz_costh_cosph - Mzr * dxdz_sinth, Mxi * dxdz_costh_cosph - Mzi * dxdz_sinth, cp, sp, LtRe, LtIm);
          ROT(-Mxr * dxdz_sinph, -Mxi * dxdz_sinph, cp, sp, LpRe, LpIm);
          const double rpr_n = (ipos - ci + 0.5) * dx * sinth * cosph + (lj - cj) * dy * sinth * sinph + (kpos - ck + 0.5) * dz * costh;
          const double cn = cos(k_wave * rpr_n), sn = sin(k_wave * rpr_n);
          ROT(JxrN * dxdz_costh_cosph - JzrN * dxdz_sinth, JxiN * dxdz_costh_cosph - JziN * dxdz_sinth, cn, sn, NtRe, NtIm);
          ROT(-JxrN * dxdz_sinph, -JxiN * dxdz_sinph, cn, sn, NpRe, NpIm);
          ROT(MxrN * dxdz_costh_cosph - MzrN * dxdz_sinth, MxiN * dxdz_costh_cosph - MziN * dxdz_sinth, cn, sn, LtRe, LtIm);
          ROT(-MxrN * dxdz_sinph, -MxiN * dxdz_sinph, cn, sn, LpRe, LpIm);
        }
      for (int ni = 0; ni < ni_ff; ni++)
        for (int nj = 0; nj < nj_ff; nj++) {
          const long p = oz + (long)ni * nj_ff + nj;
          const int ipos = (li - 1) + ni, jpos = (lj - 1) + nj;
          const double Jxr = F[CJXZP][0][p], Jxi = F[CJXZP][1][p], Jyr = F[CJYZP][0][p], Jyi = F[CJYZP][1][p];
          const double Mxr = F[CMXZP][0][p], Mxi = F[CMXZP][1][p], Myr = F[CMYZP][0][p], Myi = F[CMYZP][1][p];
          const double JxrN = F[CJXZN][0][p], JxiN = F[CJXZN][1][p], JyrN = F[CJYZN][0][p], JyiN = F[CJYZN][1][p];
          const double MxrN = F[CMXZN][0][p], MxiN = F[CMXZN][1][p], MyrN = F[CMYZN][0][p], MyiN = F[CMYZN][1][p];
          const double dxdy = dx * dy;
          const double rpr_p = (ipos - ci + 0.5) * dx * sinth * cosph + (jpos - cj + 0.5) * dy * sinth * sinph + (uk - ck) * dz * costh;
          const double cp = cos(k_wave * rpr_p), sp = sin(k_wave * rpr_p);
          const double costh_cosph = costh * cosph, costh_sinph = costh * sinph;
          const double dxdy_costh_cosph = dxdy * costh_cosph, dxdy_costh_sinph = dxdy * costh_sinph;
          const double dxdy_sinph = dxdy * sinph, dxdy_cosph = dxdy * cosph;
          ROT(Jxr * dxdy_costh_cosph + Jyr * dxdy_costh_sinph, Jxi * dxdy_costh_cosph + Jyi * dxdy_costh_sinph, cp, sp, NtRe, NtIm);
          ROT(-Jxr * dxdy_sinph + Jyr * dxdy_cosph, -Jxi * dxdy_sinph + Jyi * dxdy_cosph, cp, sp, NpRe, NpIm);
          ROT(Mxr * dxdy_costh_cosph + Myr * dxdy_costh_sinph, Mxi * dxdy_costh_cosph + Myi * dxdy_costh_sinph, cp, sp, LtRe, LtIm);
          ROT(-Mxr * dxdy_sinph + Myr * dxdy_cosph, -Mxi * dxdy_sinph + Myi * dxdy_cosph, cp, sp, LpRe, LpIm);
          const double rpr_n = (ipos - ci + 0.5) * dx * sinth * cosph + (jpos - cj + 0.5) * dy * sinth * sinph + (lk - ck) * dz * costh;
          const double cn = cos(k_wave * rpr_n), sn = sin(k_wave * rpr_n);
          ROT(JxrN * dxdy_costh_cosph + JyrN * dxdy_costh_sinph, JxiN * dxdy_costh_cosph + JyiN * dxdy_costh_sinph, cn, sn, NtRe, NtIm);
          ROT(-JxrN * dxdy_sinph + JyrN * dxdy_cosph, -JxiN * dxdy_sinph + JyiN * dxdy_cosph, cn, sn, NpRe, NpIm);
          ROT(MxrN * dxdy_costh_cosph + MyrN * dxdy_costh_sinph, MxiN * dxdy_costh_cosph + MyiN * dxdy_costh_sinph, cn, sn, LtRe, LtIm);
          ROT(-MxrN * dxdy_sinph + MyrN * dxdy_cosph, -MxiN * dxdy_sinph + MyiN * dxdy_cosph, cn, sn, LpRe, LpIm);
        }
#undef ROT
      const double LpNt_r = LpRe + ETA0 * NtRe, LpNt_i = LpIm + ETA0 * NtIm;
      dTheta[(long)mi * nA + a] = scale * (LpNt_r * LpNt_r + LpNt_i * LpNt_i);
      const double LtNp_r = LtRe - ETA0 * NpRe, LtNp_i = LtIm - ETA0 * NpIm;
      dPhi[(long)mi * nA + a] = scale * (LtNp_r * LtNp_r + LtNp_i * LtNp_i);
    }
  }
}
