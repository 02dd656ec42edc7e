/*
 * ORACLE — test infrastructure only. Never linked into, or called by, the
 * product path. Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it (through oracle/oracle.py), as the checker.
 *
 * Plain-C restatement of the QES-Winds lambda solve (reference Solver_CPU and
 * Solver_CPU_RB). Every FP32 routine reproduces the reference's expression
 * order and its float/double promotions, so that built with
 * -ffp-contract=off it agrees bit for bit with the reference sources built
 * the same way (oracle/Makefile builds both). Parity of this restatement is
 * pinned against the reference build in tests/test_oracle_pin.py and against
 * the committed golden vectors in tests/golden/.
 *
 * Grid conventions (reference src/qes/Domain.cpp:7-31, Domain.h:147-167):
 *   base counts Nx, Ny, Nz;  staggered nx = Nx+1, ny = Ny+1, nz = Nz+2;
 *   cell (i,j,k) -> i + j*(nx-1) + k*(nx-1)*(ny-1),  k in [0, nz-2];
 *   face (i,j,k) -> i + j*nx + k*nx*ny,              k in [0, nz-1];
 *   dz[k], k in [0, nz-2], dz[0] is the ghost layer below the ground.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OMEGA 1.78f /* src/winds/Solver.h:83 */

typedef struct {
  int nx, ny, nz;  /* staggered sizes */
  long X, XY;      /* cell strides */
  long FX, FXY;    /* face strides */
} grid_t;

static grid_t mkgrid(int Nx, int Ny, int Nz)
{
  grid_t g;
  g.nx = Nx + 1;
  g.ny = Ny + 1;
  g.nz = Nz + 2;
  g.X = g.nx - 1;
  g.XY = (long)(g.nx - 1) * (g.ny - 1);
  g.FX = g.nx;
  g.FXY = (long)g.nx * g.ny;
  return g;
}

static inline long cellix(const grid_t *g, int i, int j, int k) { return i + j * g->X + k * g->XY; }
static inline long faceix(const grid_t *g, int i, int j, int k) { return i + j * g->FX + k * g->FXY; }

/* Divergence of the initial field, src/winds/Solver_CPU.cpp:56-77.
 * (-2.0f * pow(alpha1, 2.0)) is a double; the x and y terms are float, the
 * m-term picks up the double literal 0.5, the n-term uses 0.5f. */
void qo_divergence(int Nx, int Ny, int Nz, float dx, float dy, const float *dz, const float *e,
                   const float *f, const float *g_, const float *h, const float *m, const float *n,
                   const float *u0, const float *v0, const float *w0, float *R)
{
  grid_t G = mkgrid(Nx, Ny, Nz);
  for (int k = 1; k < G.nz - 2; ++k)
    for (int j = 0; j < G.ny - 1; ++j)
      for (int i = 0; i < G.nx - 1; ++i) {
        long c = cellix(&G, i, j, k), fc = faceix(&G, i, j, k);
        float xt = (e[c] * u0[fc + 1] - f[c] * u0[fc]) * dx;
        float yt = (g_[c] * v0[fc + G.FX] - h[c] * v0[fc]) * dy;
        double mt = (double)(m[c] * dz[k]) * 0.5 * (double)(dz[k] + dz[k + 1]) * (double)w0[fc + G.FXY];
        float nt = n[c] * dz[k] * 0.5f * (dz[k] + dz[k - 1]) * w0[fc];
        double zt = mt - (double)nt;
        R[c] = (float)(-2.0 * ((double)(xt + yt) + zt));
      }
}

/* One SOR cell update, src/winds/Solver_CPU.cpp:107-114 (all float); the
 * reference's omega is OMEGA, other values serve the solver's over-relaxed
 * pre-phase. */
static inline float sor_cell(const grid_t *G, long c, const float *e, const float *f, const float *g_,
                             const float *h, const float *m, const float *n, const float *R, const float *L,
                             float omega)
{
  return (omega / (e[c] + f[c] + g_[c] + h[c] + m[c] + n[c])) *
             (e[c] * L[c + 1] + f[c] * L[c - 1] + g_[c] * L[c + G->X] + h[c] * L[c - G->X] +
              m[c] * L[c + G->XY] + n[c] * L[c - G->XY] - R[c]) +
         (1.0f - omega) * L[c];
}

/*
 * The reference iteration loop (Solver_CPU.cpp:86-145 for ordering 0,
 * Solver_CPU_RB.cpp:88-185 for ordering 1):
 *   while (iter < itermax && max_error > tol) {
 *     lambda_old = lambda; sweep; mirror lambda(k=0) <- lambda(k=1);
 *     max_error = max |lambda - lambda_old| over k in [1, nz-2]; ++iter; }
 * err_fp64 = 0 measures |lambda - lambda_old| in float as the reference does;
 * err_fp64 = 1 measures it in double (the solver's FP64 convergence rule).
 * err_hist (nullable) receives each iteration's error as a double.
 * Returns the number of iterations performed.
 */
/*
 * window > 0 adds the solver's window rule (no reference counterpart): after
 * an iteration that leaves the reference condition true, if the iteration
 * count is a multiple of `window`, the loop also stops when
 * max over all cells |lambda - lambda(window iterations earlier)| <= wtol,
 * in double; *stop (nullable) receives 0 (itermax), 1 (tol) or 2 (window),
 * *drift (nullable) the last window's value (-1 if none).
 */
int qo_sor_window(int ordering, int err_fp64, int Nx, int Ny, int Nz, const float *e, const float *f,
                  const float *g_, const float *h, const float *m, const float *n, const float *R, float *L,
                  float tol, int itermax, double *final_error, double *err_hist, float omega, int window,
                  double wtol, int *stop, double *drift)
{
  grid_t G = mkgrid(Nx, Ny, Nz);
  long nc = G.XY * (G.nz - 1);
  float *old = (float *)malloc(sizeof(float) * nc);
  float *snap = window > 0 ? (float *)malloc(sizeof(float) * nc) : NULL;
  if (snap) memcpy(snap, L, sizeof(float) * nc);
  int iter = 0, wstop = 0;
  double max_error = 1.0, wdrift = -1.0;
  while (iter < itermax && max_error > (double)tol && !wstop) {
    memcpy(old, L, sizeof(float) * nc);
    if (ordering == 0) {
      for (int k = 1; k < G.nz - 2; ++k)
        for (int j = 1; j < G.ny - 2; ++j)
          for (int i = 1; i < G.nx - 2; ++i) {
            long c = cellix(&G, i, j, k);
            L[c] = sor_cell(&G, c, e, f, g_, h, m, n, R, L, omega);
          }
    } else {
      for (int colour = 0; colour < 2; ++colour)
        for (int k = 1; k < G.nz - 2; ++k)
          for (int j = 1; j < G.ny - 2; ++j)
            for (int i = 1; i < G.nx - 2; ++i)
              if (((i + j + k) % 2) == colour) {
                long c = cellix(&G, i, j, k);
                L[c] = sor_cell(&G, c, e, f, g_, h, m, n, R, L, omega);
              }
    }
    for (int j = 0; j < G.ny - 1; ++j)
      for (int i = 0; i < G.nx - 1; ++i) {
        long c = cellix(&G, i, j, 0);
        L[c] = L[c + G.XY];
      }
    double me = 0.0;
    float mef = 0.0f;
    for (int k = 1; k < G.nz - 1; ++k)
      for (int j = 0; j < G.ny - 1; ++j)
        for (int i = 0; i < G.nx - 1; ++i) {
          long c = cellix(&G, i, j, k);
          if (err_fp64) {
            double d = fabs((double)L[c] - (double)old[c]);
            if (d > me) me = d;
          } else {
            float d = fabsf(L[c] - old[c]);
            if (d > mef) mef = d;
          }
        }
    max_error = err_fp64 ? me : (double)mef;
    if (err_hist) err_hist[iter] = max_error;
    iter += 1;
    if (snap && iter % window == 0 && iter < itermax && max_error > (double)tol && max_error == max_error) {
      double dw = 0.0;
      for (long c = 0; c < nc; ++c) {
        double d = fabs((double)L[c] - (double)snap[c]);
        if (d > dw || d != d) dw = d;
      }
      memcpy(snap, L, sizeof(float) * nc);
      wdrift = dw;
      if (dw <= wtol) wstop = 1;
    }
  }
  if (final_error) *final_error = max_error;
  if (stop) *stop = wstop ? 2 : (max_error > (double)tol ? 0 : 1);
  if (drift) *drift = wdrift;
  free(old);
  free(snap);
  return iter;
}

int qo_sor_omega(int ordering, int err_fp64, int Nx, int Ny, int Nz, const float *e, const float *f,
                 const float *g_, const float *h, const float *m, const float *n, const float *R, float *L,
                 float tol, int itermax, double *final_error, double *err_hist, float omega)
{
  return qo_sor_window(ordering, err_fp64, Nx, Ny, Nz, e, f, g_, h, m, n, R, L, tol, itermax, final_error,
                       err_hist, omega, 0, 0.0, NULL, NULL);
}

int qo_sor(int ordering, int err_fp64, int Nx, int Ny, int Nz, const float *e, const float *f,
           const float *g_, const float *h, const float *m, const float *n, const float *R, float *L,
           float tol, int itermax, double *final_error, double *err_hist)
{
  return qo_sor_omega(ordering, err_fp64, Nx, Ny, Nz, e, f, g_, h, m, n, R, L, tol, itermax, final_error,
                      err_hist, OMEGA);
}

/* Velocity correction and solid-cell zeroing, src/winds/Solver_CPU.cpp:157-231. */
void qo_correct(int Nx, int Ny, int Nz, float dx, float dy, const float *dz, const float *f,
                const float *h, const float *n, const int *icellflag, const float *L, const float *u0,
                const float *v0, const float *w0, float *u, float *v, float *w)
{
  grid_t G = mkgrid(Nx, Ny, Nz);
  long nf = G.FXY * G.nz;
  memcpy(u, u0, sizeof(float) * nf);
  memcpy(v, v0, sizeof(float) * nf);
  memcpy(w, w0, sizeof(float) * nf);
  const float half = 1.0f / (2.0f * 1.0f); /* (1.0f / (2.0f * (float)pow(alpha, 2.0))) */
  for (int k = 1; k < G.nz - 2; ++k)
    for (int j = 1; j < G.ny - 1; ++j)
      for (int i = 1; i < G.nx - 1; ++i) {
        long c = cellix(&G, i, j, k), fc = faceix(&G, i, j, k);
        u[fc] = u0[fc] + half * f[c] * dx * (L[c] - L[c - 1]);
      }
  for (int k = 1; k < G.nz - 2; ++k)
    for (int j = 1; j < G.ny - 1; ++j)
      for (int i = 1; i < G.nx - 1; ++i) {
        long c = cellix(&G, i, j, k), fc = faceix(&G, i, j, k);
        v[fc] = v0[fc] + half * h[c] * dy * (L[c] - L[c - G.X]);
      }
  for (int k = 1; k < G.nz - 2; ++k)
    for (int j = 1; j < G.ny - 1; ++j)
      for (int i = 1; i < G.nx - 1; ++i) {
        long c = cellix(&G, i, j, k), fc = faceix(&G, i, j, k);
        w[fc] = w0[fc] + half * n[c] * dz[k] * (L[c] - L[c - G.XY]);
      }
  for (int k = 1; k < G.nz - 1; ++k)
    for (int j = 0; j < G.ny - 1; ++j)
      for (int i = 0; i < G.nx - 1; ++i) {
        long c = cellix(&G, i, j, k), fc = faceix(&G, i, j, k);
        if (icellflag[c] == 0 || icellflag[c] == 2) {
          u[fc] = 0;
          u[fc + 1] = 0;
          v[fc] = 0;
          v[fc + G.FX] = 0;
          w[fc] = 0;
          w[fc + G.FXY] = 0;
        }
      }
}

/* ---------------------------------------------------------------------
 * FP64 run of the same red-black SOR: the same loop bounds, mirror and
 * stopping rule as qo_sor(ordering=1), with R, lambda and the correction
 * carried in double. Used to state the error of FP32 results.
 * --------------------------------------------------------------------- */
void qo_divergence_f64(int Nx, int Ny, int Nz, float dx, float dy, const float *dz, const float *e,
                       const float *f, const float *g_, const float *h, const float *m,
                       const float *n, const float *u0, const float *v0, const float *w0, double *R)
{
  grid_t G = mkgrid(Nx, Ny, Nz);
  for (int k = 1; k < G.nz - 2; ++k)
    for (int j = 0; j < G.ny - 1; ++j)
      for (int i = 0; i < G.nx - 1; ++i) {
        long c = cellix(&G, i, j, k), fc = faceix(&G, i, j, k);
        double xt = ((double)e[c] * u0[fc + 1] - (double)f[c] * u0[fc]) * dx;
        double yt = ((double)g_[c] * v0[fc + G.FX] - (double)h[c] * v0[fc]) * dy;
        double zt = (double)m[c] * dz[k] * 0.5 * ((double)dz[k] + dz[k + 1]) * w0[fc + G.FXY] -
                    (double)n[c] * dz[k] * 0.5 * ((double)dz[k] + dz[k - 1]) * w0[fc];
        R[c] = -2.0 * (xt + yt + zt);
      }
}

int qo_sor_rb_f64_omega(int Nx, int Ny, int Nz, const float *e, const float *f, const float *g_,
                        const float *h, const float *m, const float *n, const double *R, double *L,
                        double tol, int itermax, double *final_error, double om)
{
  grid_t G = mkgrid(Nx, Ny, Nz);
  long nc = G.XY * (G.nz - 1);
  double *old = (double *)malloc(sizeof(double) * nc);
  int iter = 0;
  double max_error = 1.0;
  while (iter < itermax && max_error > tol) {
    memcpy(old, L, sizeof(double) * nc);
    for (int colour = 0; colour < 2; ++colour)
      for (int k = 1; k < G.nz - 2; ++k)
        for (int j = 1; j < G.ny - 2; ++j)
          for (int i = 1; i < G.nx - 2; ++i)
            if (((i + j + k) % 2) == colour) {
              long c = cellix(&G, i, j, k);
              double s = (double)e[c] + f[c] + g_[c] + h[c] + m[c] + n[c];
              L[c] = om / s *
                         ((double)e[c] * L[c + 1] + (double)f[c] * L[c - 1] + (double)g_[c] * L[c + G.X] +
                          (double)h[c] * L[c - G.X] + (double)m[c] * L[c + G.XY] +
                          (double)n[c] * L[c - G.XY] - R[c]) +
                     (1.0 - om) * L[c];
            }
    for (int j = 0; j < G.ny - 1; ++j)
      for (int i = 0; i < G.nx - 1; ++i) {
        long c = cellix(&G, i, j, 0);
        L[c] = L[c + G.XY];
      }
    double me = 0.0;
    for (long c = G.XY; c < nc; ++c) {
      double d = fabs(L[c] - old[c]);
      if (d > me) me = d;
    }
    max_error = me;
    iter += 1;
  }
  if (final_error) *final_error = max_error;
  free(old);
  return iter;
}

int qo_sor_rb_f64(int Nx, int Ny, int Nz, const float *e, const float *f, const float *g_,
                  const float *h, const float *m, const float *n, const double *R, double *L,
                  double tol, int itermax, double *final_error)
{
  return qo_sor_rb_f64_omega(Nx, Ny, Nz, e, f, g_, h, m, n, R, L, tol, itermax, final_error, (double)OMEGA);
}

void qo_correct_f64(int Nx, int Ny, int Nz, float dx, float dy, const float *dz, const float *f,
                    const float *h, const float *n, const int *icellflag, const double *L,
                    const float *u0, const float *v0, const float *w0, double *u, double *v, double *w)
{
  grid_t G = mkgrid(Nx, Ny, Nz);
  long nf = G.FXY * G.nz;
  for (long q = 0; q < nf; ++q) {
    u[q] = u0[q];
    v[q] = v0[q];
    w[q] = w0[q];
  }
  for (int k = 1; k < G.nz - 2; ++k)
    for (int j = 1; j < G.ny - 1; ++j)
      for (int i = 1; i < G.nx - 1; ++i) {
        long c = cellix(&G, i, j, k), fc = faceix(&G, i, j, k);
        u[fc] = u0[fc] + 0.5 * f[c] * dx * (L[c] - L[c - 1]);
        v[fc] = v0[fc] + 0.5 * h[c] * dy * (L[c] - L[c - G.X]);
        w[fc] = w0[fc] + 0.5 * n[c] * dz[k] * (L[c] - L[c - G.XY]);
      }
  for (int k = 1; k < G.nz - 1; ++k)
    for (int j = 0; j < G.ny - 1; ++j)
      for (int i = 0; i < G.nx - 1; ++i) {
        long c = cellix(&G, i, j, k), fc = faceix(&G, i, j, k);
        if (icellflag[c] == 0 || icellflag[c] == 2) {
          u[fc] = u[fc + 1] = 0;
          v[fc] = v[fc + G.FX] = 0;
          w[fc] = w[fc + G.FXY] = 0;
        }
      }
}

/*
 * Discrete divergence of a face field, evaluated in double:
 *   (u[i+1]-u[i])/dx + (v[j+1]-v[j])/dy + (w[k+1]-w[k])/dz[k]
 * maximised in absolute value over fluid cells (icellflag == 1) with
 * i in [1, nx-3], j in [1, ny-3], k in [1, kmax]. kmax = nz-4 leaves out the
 * last solved layer, whose top face the reference never corrects
 * (Solver_CPU.cpp:197-209 stops at k = nz-3).
 */
double qo_max_divergence(int Nx, int Ny, int Nz, float dx, float dy, const float *dz,
                         const int *icellflag, const float *u, const float *v, const float *w, int kmax)
{
  grid_t G = mkgrid(Nx, Ny, Nz);
  double mx = 0.0;
  for (int k = 1; k <= kmax; ++k)
    for (int j = 1; j < G.ny - 2; ++j)
      for (int i = 1; i < G.nx - 2; ++i) {
        long c = cellix(&G, i, j, k), fc = faceix(&G, i, j, k);
        if (icellflag[c] != 1) continue;
        double d = ((double)u[fc + 1] - u[fc]) / dx + ((double)v[fc + G.FX] - v[fc]) / dy +
                   ((double)w[fc + G.FXY] - w[fc]) / dz[k];
        if (fabs(d) > mx) mx = fabs(d);
      }
  return mx;
}

/* Log-law wall treatment of the stair-step walls: the list construction of
 * Wall::defineWalls (src/winds/Wall.cpp:287-340: fluid cells, k in [1, nz-3],
 * loop order k, i, j, neighbours by flat cell index as Domain::cellAdd takes
 * them) followed by the six list loops of Wall::wallLogBC
 * (src/winds/Wall.cpp:656-796), in place on u0, v0, w0. Wall.h includes
 * <math.h> under `using namespace std`, so atan2, log, cos and sin of floats
 * are the float functions, and sqrt(pow(x, 2.0) + ...) is evaluated in double.
 * dxy is Domain::getDomainSize()'s first value, which the reference uses for
 * both the x and the y walls (it returns dx twice, src/qes/Domain.h:104); dz is
 * its third, the Domain's nominal dz. vk = 0.4f (WINDSGeneralData.h).
 * Returns -1, changing nothing, when a cell in that k range carries a cut-cell
 * flag (7 or 8), whose walls the first part of wallLogBC treats; else 0. */
static int wl_solid(int f) { return f == 0 || f == 2; }

static void wl_fix(float *a, float *b, float *c_normal, long f, long nb, float d1, float d2, float z0)
{
  /* a, b: the two wall-parallel components (wind_dir = atan2(b, a)); the
   * normal component c_normal is zeroed. */
  const float vk = 0.4f;
  float ustar_wall = 0.1f, wind_dir = 0.0f, vel_mag1 = 0.0f, vel_mag2, new_ustar;
  for (int iter = 0; iter < 20; iter++) {
    wind_dir = atan2f(b[nb], a[nb]);
    vel_mag2 = (float)sqrt(pow(a[nb], 2.0) + pow(b[nb], 2.0));
    vel_mag1 = vel_mag2 - (ustar_wall / vk) * logf(d2 / d1);
    c_normal[f] = 0;
    a[f] = vel_mag1 * cosf(wind_dir);
    b[f] = vel_mag1 * sinf(wind_dir);
    new_ustar = vk * vel_mag1 / logf(d1 / z0);
    ustar_wall = new_ustar;
  }
}

int qo_wall_log(int Nx, int Ny, int Nz, float dxy, float dz, float z0, const int *flag, float *u0, float *v0,
                float *w0)
{
  grid_t g = mkgrid(Nx, Ny, Nz);
  for (int k = 1; k < g.nz - 2; k++)
    for (int i = 0; i < g.nx - 1; i++)
      for (int j = 0; j < g.ny - 1; j++) {
        const int fl = flag[cellix(&g, i, j, k)];
        if (fl == 7 || fl == 8) return -1;
      }
  for (int side = 0; side < 6; side++) {
    /* below, above (0.5 dz), back, front (0.5 dx), right, left (0.5 "dy" = dx) */
    const float d1 = side < 2 ? 0.5f * dz : 0.5f * dxy, d2 = side < 2 ? 1.5f * dz : 1.5f * dxy;
    for (int k = 1; k < g.nz - 2; k++)
      for (int i = 0; i < g.nx - 1; i++)
        for (int j = 0; j < g.ny - 1; j++) {
          const long c = cellix(&g, i, j, k), f = faceix(&g, i, j, k);
          const int fl = flag[c];
          if (fl == 0 || fl == 2) continue;
          switch (side) {
          case 0:
            if (wl_solid(flag[c - g.XY])) wl_fix(u0, v0, w0, f, f + g.FXY, d1, d2, z0);
            break;
          case 1:
            if (wl_solid(flag[c + g.XY])) wl_fix(u0, v0, w0, f, f - g.FXY, d1, d2, z0);
            break;
          case 2:
            if (wl_solid(flag[c - 1]) && i > 0) wl_fix(v0, w0, u0, f, f + 1, d1, d2, z0);
            break;
          case 3:
            if (wl_solid(flag[c + 1])) wl_fix(v0, w0, u0, f, f - 1, d1, d2, z0);
            break;
          case 4:
            if (wl_solid(flag[c - g.X]) && j > 0) wl_fix(u0, w0, v0, f, f + g.FX, d1, d2, z0);
            break;
          default:
            if (wl_solid(flag[c + g.X])) wl_fix(u0, w0, v0, f, f - g.FX, d1, d2, z0);
            break;
          }
        }
  }
  return 0;
}

/* -------------------------------------------------------------------------
 * Seeded synthetic city, restated for the reference-only benchmark leg: the
 * same cities the product's generator (qesb_city_random / qesb_city_build)
 * makes, built without the product library. The wall coefficients and the
 * solid-face zeroing then come from the reference's own Wall.cpp
 * (oracle/_ref); this file supplies what the reference has no code for: the
 * seeded building layout, the cell flags of the buildings (PolyBuilding's
 * PNPOLY test, src/winds/PolyBuilding.cpp:157-224, for the closed 5-vertex
 * ring of RectangularBuilding.h:70-108) and the power-law inflow
 * (WindProfilerSensorType.cpp:220,328-333).
 * ------------------------------------------------------------------------- */

/* SplitMix64 (Steele, Lea, Flood 2014). */
static uint64_t sm64_next(uint64_t *s)
{
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static float sm64_uniform(uint64_t *s, float a, float b)
{
  double u = (double)(sm64_next(s) >> 11) * (1.0 / 9007199254740992.0);
  return (float)(a + (b - a) * u);
}

/* Buildings (x_start, y_start, length, width, height, base_height: 6 floats
 * each) and inflow (u_ref, z_ref, p, dir_deg) of the seed's city: up to
 * max_b non-overlapping cuboids with a one-cell gap, kept a margin from the
 * domain edges, placed by rejection. Returns the count. */
int qo_city_random(int Nx, int Ny, float dx, float dy, uint64_t seed, int max_b, float fp_min, float fp_max,
                   float h_min, float h_max, float *b, float *inflow)
{
  uint64_t s = seed;
  const float Lx = Nx * dx, Ly = Ny * dy;
  const float dmax = dx > dy ? dx : dy;
  const float margin = 2.0f * dmax + 1.0f, gap = dmax;
  int nb = 0;
  for (int attempt = 0; attempt < 200 * max_b && nb < max_b; ++attempt) {
    float len = sm64_uniform(&s, fp_min, fp_max);
    float wid = sm64_uniform(&s, fp_min, fp_max);
    float hgt = sm64_uniform(&s, h_min, h_max);
    if (Lx - 2 * margin - len <= 0 || Ly - 2 * margin - wid <= 0) continue;
    float xs = floorf(sm64_uniform(&s, margin, Lx - margin - len));
    float ys = floorf(sm64_uniform(&s, margin, Ly - margin - wid));
    int ok = 1;
    for (int q = 0; q < nb && ok; ++q) {
      const float *o = b + 6 * q;
      if (xs < o[0] + o[2] + gap && o[0] < xs + len + gap && ys < o[1] + o[3] + gap && o[1] < ys + wid + gap) ok = 0;
    }
    if (ok) {
      float *c = b + 6 * nb++;
      c[0] = xs;
      c[1] = ys;
      c[2] = len;
      c[3] = wid;
      c[4] = hgt;
      c[5] = 0.0f;
    }
  }
  inflow[0] = sm64_uniform(&s, 3.0f, 10.0f);
  inflow[1] = 10.0f;
  inflow[2] = sm64_uniform(&s, 0.1f, 0.3f);
  inflow[3] = sm64_uniform(&s, 0.0f, 360.0f);
  return nb;
}

/* z and z_face from dz, as Domain::defineVerticalGrid (src/qes/Domain.cpp:135-151). */
static void vgrid(int nz, const float *dz, float *z, float *zf)
{
  zf[0] = -dz[0];
  zf[1] = 0.0f;
  for (int k = 2; k < nz; ++k) zf[k] = zf[k - 1] + dz[k - 1];
  z[0] = -0.5f * dz[0];
  for (int k = 1; k < nz - 1; ++k) z[k] = 0.5f * (zf[k] + zf[k + 1]);
}

/* icellflag of the city: 1 everywhere, 2 on the ground plane k = 0
 * (WINDSGeneralData.cpp:438-444), 0 in the buildings' cells. */
void qo_city_flags(int Nx, int Ny, int Nz, float dx, float dy, const float *dz, int nb, const float *b, int *flag)
{
  grid_t G = mkgrid(Nx, Ny, Nz);
  const long nc = G.XY * (G.nz - 1);
  float *z = (float *)malloc(sizeof(float) * (G.nz - 1)), *zf = (float *)malloc(sizeof(float) * G.nz);
  vgrid(G.nz, dz, z, zf);
  for (long c = 0; c < nc; ++c) flag[c] = 1;
  for (int j = 0; j < G.ny - 1; ++j)
    for (int i = 0; i < G.nx - 1; ++i) flag[cellix(&G, i, j, 0)] = 2;
  for (int q = 0; q < nb; ++q) {
    const float *B = b + 6 * q;
    const float xs = B[0], ys = B[1], len = B[2], wid = B[3], hgt = B[4], base = B[5];
    float px[5], py[5];
    px[0] = px[4] = xs;
    py[0] = py[4] = ys;
    px[1] = xs - wid * 0.0f;
    py[1] = ys + wid * 1.0f;
    px[2] = px[1] + len * 1.0f;
    py[2] = py[1] + len * 0.0f;
    px[3] = xs + len * 1.0f;
    py[3] = ys + len * 0.0f;
    float x_min = px[0], x_max = px[0], y_min = py[0], y_max = py[0];
    for (int v = 1; v < 5; ++v) {
      if (px[v] > x_max) x_max = px[v];
      if (px[v] < x_min) x_min = px[v];
      if (py[v] > y_max) y_max = py[v];
      if (py[v] < y_min) y_min = py[v];
    }
    const int i_start = (int)(x_min / dx), i_end = (int)((x_max / dx) + 1);
    const int j_start = (int)(y_min / dy), j_end = (int)((y_max / dy) + 1);
    const float top = hgt + base;
    int k_start = 1, k_end = 1;
    for (int k = 1; k < G.nz - 1; ++k) {
      k_start = k;
      if (base <= zf[k + 1]) break;
    }
    for (int k = 0; k < G.nz - 1; ++k) {
      k_end = k + 1;
      if (top < z[k + 1]) break;
    }
    for (int j = j_start; j <= j_end; ++j) {
      const float yc = (float)((j + 0.5) * dy);
      for (int i = i_start; i <= i_end; ++i) {
        const float xc = (float)((i + 0.5) * dx);
        unsigned v = 0, st = 0;
        int cross = 0;
        while (v < 4) {
          if ((py[v] <= yc && py[v + 1] > yc) || (py[v] > yc && py[v + 1] <= yc)) {
            const float t = (yc - py[v]) / (py[v + 1] - py[v]);
            if (xc < (px[v] + t * (px[v + 1] - px[v]))) cross += 1;
          }
          v += 1;
          if (px[v] == px[st] && py[v] == py[st]) {
            v += 1;
            st = v;
          }
        }
        if (cross % 2 != 0 && i >= 0 && j >= 0 && i < G.X && j < G.ny - 1)
          for (int k = k_start; k < k_end && k < G.nz - 1; ++k) flag[cellix(&G, i, j, k)] = 0;
      }
    }
  }
  free(z);
  free(zf);
}

/* Power-law inflow on every face column, faces k in [1, nz-2]; w0 = 0
 * (flat terrain, one sensor). Solid faces are not zeroed here. */
void qo_city_inflow(int Nx, int Ny, int Nz, const float *dz, const float *inflow, float *u0, float *v0, float *w0)
{
  grid_t G = mkgrid(Nx, Ny, Nz);
  const long nf = G.FXY * G.nz;
  float *z = (float *)malloc(sizeof(float) * (G.nz - 1)), *zf = (float *)malloc(sizeof(float) * G.nz);
  vgrid(G.nz, dz, z, zf);
  memset(u0, 0, sizeof(float) * nf);
  memset(v0, 0, sizeof(float) * nf);
  memset(w0, 0, sizeof(float) * nf);
  const float theta = (float)((270.0 - inflow[3]) * M_PI / 180.0);
  for (int k = 1; k < G.nz - 1; ++k) {
    const float s = powf((z[k] - 0.0f) / inflow[1], inflow[2]);
    const float up = cosf(theta) * inflow[0] * s, vp = sinf(theta) * inflow[0] * s;
    for (int j = 0; j < G.ny; ++j)
      for (int i = 0; i < G.nx; ++i) {
        const long q = faceix(&G, i, j, k);
        u0[q] = up;
        v0[q] = vp;
      }
  }
  free(z);
  free(zf);
}
