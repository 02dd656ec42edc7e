// Seeded synthetic-city generator: the solver inputs for flat terrain,
// stair-step cuboid buildings and a single power-law inflow profile.
//
// Each stage restates a reference set-up step for this subset of inputs
// (no terrain, no cut cells, no parameterizations):
//   qesb_city_dz      Domain::defineVerticalStretching/defineVerticalGrid
//                     (src/qes/Domain.cpp:121-151)
//   ground flags      WINDSGeneralData.cpp:438-444 (k = 0 plane is terrain, flag 2)
//   building cells    PolyBuilding::setCellFlags (src/winds/PolyBuilding.cpp:130-237)
//                     for the 5-vertex polygon of RectangularBuilding.h:70-108
//   wall coefficients Wall::defineWalls + Wall::solverCoefficients
//                     (src/winds/Wall.cpp:44-350, 827-846) for flags {0, 1, 2}
//   inflow            WindProfilerSensorType.cpp:220 (theta), :328-333 (power law),
//                     :571-621 (single-sensor fill over all faces)
//   solid faces       Wall::setVelocityZero (src/winds/Wall.cpp:805-825)
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "qesb.h"
#include "qesb_internal.h"

namespace {

struct Grid {
  int nx, ny, nz;
  long X, XY, FX, FXY;
  Grid(const qesb_grid &g)
      : nx(g.Nx + 1), ny(g.Ny + 1), nz(g.Nz + 2), X(g.Nx), XY((long)g.Nx * g.Ny), FX(g.Nx + 1),
        FXY((long)(g.Nx + 1) * (g.Ny + 1))
  {
  }
  long cell(int i, int j, int k) const { return i + j * X + k * XY; }
  long face(int i, int j, int k) const { return i + j * FX + k * FXY; }
  long ncell() const { return XY * (nz - 1); }
  long nface() const { return FXY * nz; }
};

inline bool solid(int flag) { return flag == 0 || flag == 2; }

// z and z_face from dz_array, Domain::defineVerticalGrid (Domain.cpp:135-151).
void vertical_grid(const Grid &G, const float *dz, std::vector<float> &z, std::vector<float> &zf)
{
  zf.assign(G.nz, 0.0f);
  zf[0] = -dz[0];
  zf[1] = 0.0f;
  for (int k = 2; k < G.nz; ++k) zf[k] = zf[k - 1] + dz[k - 1];
  z.assign(G.nz - 1, 0.0f);
  z[0] = -0.5f * dz[0];
  for (int k = 1; k < G.nz - 1; ++k) z[k] = 0.5f * (zf[k] + zf[k + 1]);
}

// PolyBuilding::setCellFlags for an unrotated rectangle. The polygon is the
// closed 5-vertex ring that RectangularBuilding builds; the inside test is
// the PNPOLY crossing count on cell centres, with the reference's float
// arithmetic.
void rasterise(const Grid &G, float dx, float dy, const std::vector<float> &z,
               const std::vector<float> &zf, const qesb_building &b, int *flag)
{
  float xs = b.x_start, ys = b.y_start;
  float px[5], py[5];
  px[0] = px[4] = xs;
  py[0] = py[4] = ys;
  px[1] = xs - b.width * 0.0f;
  py[1] = ys + b.width * 1.0f;
  px[2] = px[1] + b.length * 1.0f;
  py[2] = py[1] + b.length * 0.0f;
  px[3] = xs + b.length * 1.0f;
  py[3] = ys + b.length * 0.0f;
  float x_min = px[0], x_max = px[0], y_min = py[0], y_max = py[0];
  for (int q = 1; q < 5; ++q) {
    x_max = std::max(x_max, px[q]);
    x_min = std::min(x_min, px[q]);
    y_max = std::max(y_max, py[q]);
    y_min = std::min(y_min, py[q]);
  }
  int i_start = (int)(x_min / dx), i_end = (int)((x_max / dx) + 1);
  int j_start = (int)(y_min / dy), j_end = (int)((y_max / dy) + 1);
  float height_eff = b.height + b.base_height;
  int k_start = 1, k_end = 1;
  for (int k = 1; k < (int)z.size(); ++k) {
    k_start = k;
    if (b.base_height <= zf[k + 1]) break;
  }
  for (int k = 0; k < (int)z.size(); ++k) {
    k_end = k + 1;
    if (height_eff < z[k + 1]) break;
  }
  for (int j = j_start; j <= j_end; ++j) {
    float y_cent = (float)((j + 0.5) * dy);
    for (int i = i_start; i <= i_end; ++i) {
      float x_cent = (float)((i + 0.5) * dx);
      unsigned vert = 0, start = 0;
      int crossings = 0;
      while (vert < 4) {
        if ((py[vert] <= y_cent && py[vert + 1] > y_cent) || (py[vert] > y_cent && py[vert + 1] <= y_cent)) {
          float t = (y_cent - py[vert]) / (py[vert + 1] - py[vert]);
          if (x_cent < (px[vert] + t * (px[vert + 1] - px[vert]))) crossings += 1;
        }
        vert += 1;
        if (px[vert] == px[start] && py[vert] == py[start]) {
          vert += 1;
          start = vert;
        }
      }
      if (crossings % 2 != 0 && i >= 0 && j >= 0 && i < G.X && j < G.XY / G.X) {
        for (int k = k_start; k < k_end && k < G.nz - 1; ++k) flag[G.cell(i, j, k)] = 0;
      }
    }
  }
}

// Wall::defineWalls restricted to flags {0, 1, 2}, all volume fractions 1.
// With those inputs the clamps, the cut-cell branches and the all-zero
// fix-ups are no-ops; what remains is: a non-solid cell in k in [1, nz-3]
// loses the coefficient toward each solid neighbour. Neighbours are found
// by linear-index offsets exactly as Domain::cellAdd does, so at the x and
// y edges the "+1" neighbour is the first cell of the next row / plane; the
// "-1" neighbours are guarded by i > 0 and j > 0 as in Wall.cpp:143-157.
// Then Wall::solverCoefficients divides by dx*dx for e, f and, because
// Domain::getDomainSize returns dx twice (src/qes/Domain.h:104), also for g, h.
void walls(const Grid &G, float dx, const float *dz, const int *flag, float *e, float *f, float *g,
           float *h, float *m, float *n)
{
  const long nc = G.ncell();
  for (long c = 0; c < nc; ++c) e[c] = f[c] = g[c] = h[c] = m[c] = n[c] = 1.0f;
  for (int k = 1; k < G.nz - 2; ++k)
    for (int i = 0; i < G.nx - 1; ++i)
      for (int j = 0; j < G.ny - 1; ++j) {
        long c = G.cell(i, j, k);
        if (solid(flag[c])) continue;
        if (solid(flag[c - G.XY])) n[c] = 0.0f;
        if (solid(flag[c + G.XY])) m[c] = 0.0f;
        if (solid(flag[c - 1]) && i > 0) f[c] = 0.0f;
        if (solid(flag[c + 1])) e[c] = 0.0f;
        if (solid(flag[c - G.X]) && j > 0) h[c] = 0.0f;
        if (solid(flag[c + G.X])) g[c] = 0.0f;
      }
  const float dy_eff = dx;
  for (int k = 1; k < G.nz - 2; ++k) {
    const float dm = dz[k] * 0.5f * (dz[k] + dz[k + 1]);
    const float dn = dz[k] * 0.5f * (dz[k] + dz[k - 1]);
    for (int j = 0; j < G.ny - 1; ++j)
      for (int i = 0; i < G.nx - 1; ++i) {
        long c = G.cell(i, j, k);
        e[c] = e[c] / (dx * dx);
        f[c] = f[c] / (dx * dx);
        g[c] = g[c] / (dy_eff * dy_eff);
        h[c] = h[c] / (dy_eff * dy_eff);
        m[c] = m[c] / dm;
        n[c] = n[c] / dn;
      }
  }
}

// Single-sensor power-law profile on flat terrain: every face column gets
// u_prof[k] for k in [1, nz-2], w0 = 0 (terrain_face_id = 1 everywhere, so
// every branch of singleSensorInterpolation picks u_prof[k]).
void inflow(const Grid &G, const std::vector<float> &z, const qesb_inflow &in, float *u0, float *v0,
            float *w0)
{
  const long nf = G.nface();
  std::memset(u0, 0, sizeof(float) * nf);
  std::memset(v0, 0, sizeof(float) * nf);
  std::memset(w0, 0, sizeof(float) * nf);
  const float theta = (float)((270.0 - in.dir_deg) * M_PI / 180.0);
  const float z_terrain = 0.0f;
  for (int k = 1; k < G.nz - 1; ++k) {
    const float s = std::pow((z[k] - z_terrain) / in.z_ref, in.p);
    const float up = std::cos(theta) * in.u_ref * s;
    const float vp = std::sin(theta) * in.u_ref * s;
    for (int j = 0; j < G.ny; ++j)
      for (int i = 0; i < G.nx; ++i) {
        long q = G.face(i, j, k);
        u0[q] = up;
        v0[q] = vp;
        w0[q] = 0.0f;
      }
  }
}

void velocity_zero(const Grid &G, const int *flag, float *u0, float *v0, float *w0)
{
  for (int k = 0; k < G.nz - 1; ++k)
    for (int j = 1; j < G.ny - 1; ++j)
      for (int i = 1; i < G.nx - 1; ++i) {
        long c = G.cell(i, j, k), q = G.face(i, j, k);
        if (solid(flag[c])) {
          u0[q] = 0.0f;
          u0[q + 1] = 0.0f;
          v0[q] = 0.0f;
          v0[q + G.FX] = 0.0f;
          w0[q] = 0.0f;
          w0[q + G.FXY] = 0.0f;
        }
      }
}

// SplitMix64 (Steele, Lea, Flood 2014): one 64-bit state, one output per step.
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next()
  {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  float uniform(float a, float b) { return (float)(a + (b - a) * uniform()); }
};

bool valid_grid(const qesb_grid *g)
{
  return g && g->Nx >= 3 && g->Ny >= 3 && g->Nz >= 2 && g->dx > 0 && g->dy > 0 && g->dz_array;
}

}  // namespace

extern "C" {

qesb_status qesb_city_dz(int Nz, float dz0, float ratio, float *dz_array)
{
  if (Nz < 1 || !(dz0 > 0) || !(ratio > 0) || !dz_array) return qesb_fail(QESB_ERR_ARG, "qesb_city_dz: bad arguments");
  double d = dz0;
  for (int k = 1; k <= Nz; ++k) {
    dz_array[k] = (float)d;
    d *= ratio;
  }
  dz_array[0] = dz_array[1];
  return QESB_OK;
}

qesb_status qesb_city_build(const qesb_grid *grid, int n_buildings, const qesb_building *b,
                            const qesb_inflow *in, int *icellflag, float *e, float *f, float *g,
                            float *hc, float *m, float *n, float *u0, float *v0, float *w0)
{
  if (!valid_grid(grid) || n_buildings < 0 || (n_buildings > 0 && !b) || !in || !icellflag || !e ||
      !f || !g || !hc || !m || !n || !u0 || !v0 || !w0)
    return qesb_fail(QESB_ERR_ARG, "qesb_city_build: bad arguments");
  Grid G(*grid);
  std::vector<float> z, zf;
  vertical_grid(G, grid->dz_array, z, zf);
  const long nc = G.ncell();
  for (long c = 0; c < nc; ++c) icellflag[c] = 1;
  for (int j = 0; j < G.ny - 1; ++j)
    for (int i = 0; i < G.nx - 1; ++i) icellflag[G.cell(i, j, 0)] = 2;
  for (int q = 0; q < n_buildings; ++q) rasterise(G, grid->dx, grid->dy, z, zf, b[q], icellflag);
  walls(G, grid->dx, grid->dz_array, icellflag, e, f, g, hc, m, n);
  inflow(G, z, *in, u0, v0, w0);
  velocity_zero(G, icellflag, u0, v0, w0);
  return QESB_OK;
}

qesb_status qesb_city_inflow(const qesb_grid *grid, const int *icellflag, const qesb_inflow *in, float *u0,
                             float *v0, float *w0)
{
  if (!valid_grid(grid) || !icellflag || !in || !u0 || !v0 || !w0)
    return qesb_fail(QESB_ERR_ARG, "qesb_city_inflow: bad arguments");
  Grid G(*grid);
  std::vector<float> z, zf;
  vertical_grid(G, grid->dz_array, z, zf);
  inflow(G, z, *in, u0, v0, w0);
  velocity_zero(G, icellflag, u0, v0, w0);
  return QESB_OK;
}

qesb_status qesb_city_random(const qesb_grid *grid, uint64_t seed, int max_buildings, float fp_min,
                             float fp_max, float h_min, float h_max, qesb_building *b_out,
                             int *n_out, qesb_inflow *inflow_out)
{
  if (!valid_grid(grid) || max_buildings < 0 || (max_buildings > 0 && !b_out) || !n_out ||
      !inflow_out || !(fp_min > 0) || fp_max < fp_min || h_max < h_min)
    return qesb_fail(QESB_ERR_ARG, "qesb_city_random: bad arguments");
  SplitMix64 rng(seed);
  const float Lx = grid->Nx * grid->dx, Ly = grid->Ny * grid->dy;
  const float margin = 2.0f * std::max(grid->dx, grid->dy) + 1.0f;
  const float gap = std::max(grid->dx, grid->dy);
  int nb = 0;
  for (int attempt = 0; attempt < 200 * max_buildings && nb < max_buildings; ++attempt) {
    qesb_building c;
    c.length = rng.uniform(fp_min, fp_max);
    c.width = rng.uniform(fp_min, fp_max);
    c.height = rng.uniform(h_min, h_max);
    c.base_height = 0.0f;
    if (Lx - 2 * margin - c.length <= 0 || Ly - 2 * margin - c.width <= 0) continue;
    c.x_start = std::floor(rng.uniform(margin, Lx - margin - c.length));
    c.y_start = std::floor(rng.uniform(margin, Ly - margin - c.width));
    bool ok = true;
    for (int q = 0; q < nb && ok; ++q) {
      const qesb_building &o = b_out[q];
      if (c.x_start < o.x_start + o.length + gap && o.x_start < c.x_start + c.length + gap &&
          c.y_start < o.y_start + o.width + gap && o.y_start < c.y_start + c.width + gap)
        ok = false;
    }
    if (ok) b_out[nb++] = c;
  }
  *n_out = nb;
  inflow_out->u_ref = rng.uniform(3.0f, 10.0f);
  inflow_out->z_ref = 10.0f;
  inflow_out->p = rng.uniform(0.1f, 0.3f);
  inflow_out->dir_deg = rng.uniform(0.0f, 360.0f);
  return QESB_OK;
}

}  // extern "C"
