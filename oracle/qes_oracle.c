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
int qo_sor_omega(int ordering, int err_fp64, int Nx, int Ny, int Nz, const float *e, const float *f,
                 const float *g_, const float *h, const float *m, const float *n, const float *R, float *L,
                 float tol, int itermax, double *final_error, double *err_hist, float omega)
{
  grid_t G = mkgrid(Nx, Ny, Nz);
  long nc = G.XY * (G.nz - 1);
  float *old = (float *)malloc(sizeof(float) * nc);
  int iter = 0;
  double max_error = 1.0;
  while (iter < itermax && max_error > (double)tol) {
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
  }
  if (final_error) *final_error = max_error;
  free(old);
  return iter;
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
