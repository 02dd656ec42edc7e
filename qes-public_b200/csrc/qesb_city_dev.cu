// Device-side set-up of the solver inputs for synthetic cities: the same
// flags, wall coefficients and initial winds as qesb_city_build
// (qesb_city.cpp), written by kernels into device arrays, so an ensemble of
// cities or wind directions goes from a building list to a solve without a
// host round trip. Compiled with -fmad=false: the point-in-polygon test and
// the coefficient divisions round exactly as the host generator's.
//
// Stages (the reference set-up step each restates):
//   k_city_flags_init  all cells 1, the k = 0 plane 2 (terrain)
//                      (WINDSGeneralData.cpp:438-444)
//   k_city_flags_bld   one block per building: cells whose centre passes the
//                      PNPOLY crossing test, k in [k_start, k_end), set to 0
//                      (PolyBuilding::setCellFlags, PolyBuilding.cpp:130-237)
//   k_city_walls       a non-solid cell in k in [1, nz-3] drops the
//                      coefficient toward each solid neighbour, found by
//                      linear-index offsets as Domain::cellAdd does; then
//                      the division by dx^2 (e, f, and g, h through the
//                      reference's dx-for-dy) and the z metric
//                      (Wall.cpp:44-350, 827-846)
//   k_city_winds       power-law column profile on every face, w0 = 0, then
//                      the faces of solid cells zeroed (gathered per face)
//                      (WindProfilerSensorType.cpp:220, 328-333, 571-621;
//                      Wall::setVelocityZero, Wall.cpp:805-825)
// The vertical grid, the per-building boxes and k ranges, and the profile
// (std::pow, cos, sin of the host) are evaluated on the host exactly as
// qesb_city_build does and uploaded with the launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "qesb.h"
#include "qesb_internal.h"

namespace {

#define CK(x)                                                                                   \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

struct CityGrid {
  int nx, ny, nz;
  long X, XY, FX, FXY;
  __host__ __device__ long cell(int i, int j, int k) const { return i + j * X + k * XY; }
  __host__ __device__ long face(int i, int j, int k) const { return i + j * FX + k * FXY; }
};

// One building as the device sees it: the closed 5-vertex ring, the cell box
// and the layer range, all computed on the host.
struct DevBuilding {
  float px[5], py[5];
  int i_start, i_end, j_start, j_end, k_start, k_end;
};

__device__ __forceinline__ bool solid(int flag) { return flag == 0 || flag == 2; }

__global__ void k_city_flags_init(CityGrid G, int *flag)
{
  const long nc = G.XY * (G.nz - 1);
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < nc; c += (long)gridDim.x * blockDim.x)
    flag[c] = c < G.XY ? 2 : 1;
}

__global__ void k_city_flags_bld(CityGrid G, float dx, float dy, const DevBuilding *__restrict__ bld, int *flag)
{
  const DevBuilding b = bld[blockIdx.x];
  const int ni = b.i_end - b.i_start + 1, nj = b.j_end - b.j_start + 1;
  const int Y = (int)(G.XY / G.X);
  for (int t = threadIdx.x; t < ni * nj; t += blockDim.x) {
    const int j = b.j_start + t / ni, i = b.i_start + t % ni;
    const float y_cent = (float)((j + 0.5) * dy);
    const float x_cent = (float)((i + 0.5) * dx);
    unsigned vert = 0, start = 0;
    int crossings = 0;
    while (vert < 4) {
      if ((b.py[vert] <= y_cent && b.py[vert + 1] > y_cent) || (b.py[vert] > y_cent && b.py[vert + 1] <= y_cent)) {
        const float tt = (y_cent - b.py[vert]) / (b.py[vert + 1] - b.py[vert]);
        if (x_cent < (b.px[vert] + tt * (b.px[vert + 1] - b.px[vert]))) crossings += 1;
      }
      vert += 1;
      if (b.px[vert] == b.px[start] && b.py[vert] == b.py[start]) {
        vert += 1;
        start = vert;
      }
    }
    if (crossings % 2 != 0 && i >= 0 && j >= 0 && i < G.X && j < Y)
      for (int k = b.k_start; k < b.k_end && k < G.nz - 1; ++k) flag[G.cell(i, j, k)] = 0;
  }
}

__global__ void k_city_walls(CityGrid G, float dx, const float *__restrict__ dz, const int *__restrict__ flag,
                             float *__restrict__ e, float *__restrict__ f, float *__restrict__ g,
                             float *__restrict__ h, float *__restrict__ m, float *__restrict__ n)
{
  const int j = blockIdx.y, k = blockIdx.z;
  for (int i = threadIdx.x; i < G.nx - 1; i += blockDim.x) {
    const long c = G.cell(i, j, k);
    float ce = 1.0f, cf = 1.0f, cg = 1.0f, chh = 1.0f, cm = 1.0f, cn = 1.0f;
    if (k >= 1 && k < G.nz - 2) {
      if (!solid(flag[c])) {
        if (solid(flag[c - G.XY])) cn = 0.0f;
        if (solid(flag[c + G.XY])) cm = 0.0f;
        if (solid(flag[c - 1]) && i > 0) cf = 0.0f;
        if (solid(flag[c + 1])) ce = 0.0f;
        if (solid(flag[c - G.X]) && j > 0) chh = 0.0f;
        if (solid(flag[c + G.X])) cg = 0.0f;
      }
      const float dm = dz[k] * 0.5f * (dz[k] + dz[k + 1]);
      const float dn = dz[k] * 0.5f * (dz[k] + dz[k - 1]);
      const float dy_eff = dx;
      ce = ce / (dx * dx);
      cf = cf / (dx * dx);
      cg = cg / (dy_eff * dy_eff);
      chh = chh / (dy_eff * dy_eff);
      cm = cm / dm;
      cn = cn / dn;
    }
    e[c] = ce;
    f[c] = cf;
    g[c] = cg;
    h[c] = chh;
    m[c] = cm;
    n[c] = cn;
  }
}

// Cell (i, j, k) as Wall::setVelocityZero visits it: i in [1, nx-2],
// j in [1, ny-2], k in [0, nz-2], and solid.
__device__ __forceinline__ bool zeroing_cell(const CityGrid &G, const int *flag, int i, int j, int k)
{
  return i >= 1 && i <= G.nx - 2 && j >= 1 && j <= G.ny - 2 && k >= 0 && k <= G.nz - 2 &&
         solid(flag[G.cell(i, j, k)]);
}

__global__ void k_city_winds(CityGrid G, const float *__restrict__ up, const float *__restrict__ vp,
                             const int *__restrict__ flag, float *__restrict__ u0, float *__restrict__ v0,
                             float *__restrict__ w0)
{
  const int j = blockIdx.y, k = blockIdx.z;
  const bool col = k >= 1 && k <= G.nz - 2;
  const float uk = col ? up[k] : 0.0f, vk = col ? vp[k] : 0.0f;
  for (int i = threadIdx.x; i < G.nx; i += blockDim.x) {
    const long q = G.face(i, j, k);
    float uu = uk, vv = vk, ww = 0.0f;
    if (zeroing_cell(G, flag, i, j, k) || zeroing_cell(G, flag, i - 1, j, k)) uu = 0.0f;
    if (zeroing_cell(G, flag, i, j, k) || zeroing_cell(G, flag, i, j - 1, k)) vv = 0.0f;
    (void)ww;
    u0[q] = uu;
    v0[q] = vv;
    w0[q] = 0.0f;
  }
}

}  // namespace

qesb_status qesb_city_walls_dev(int Nx, int Ny, int Nz, float dx, const float *d_dz, const int *d_flag, float *e,
                                float *f, float *g, float *hc, float *m, float *n, void *stream)
{
  CityGrid G;
  G.nx = Nx + 1;
  G.ny = Ny + 1;
  G.nz = Nz + 2;
  G.X = Nx;
  G.XY = (long)Nx * Ny;
  G.FX = Nx + 1;
  G.FXY = (long)(Nx + 1) * (Ny + 1);
  k_city_walls<<<dim3(1, G.ny - 1, G.nz - 1), 256, 0, static_cast<cudaStream_t>(stream)>>>(G, dx, d_dz, d_flag, e, f, g,
                                                                                           hc, m, n);
  const cudaError_t ce = cudaGetLastError();
  return ce == cudaSuccess ? QESB_OK : qesb_fail(QESB_ERR_CUDA, "wall coefficients: %s", cudaGetErrorString(ce));
}

extern "C" qesb_status qesb_city_build_device(const qesb_grid *grid, int n_buildings, const qesb_building *b,
                                              const qesb_inflow *in, int *icellflag, float *e, float *f,
                                              float *g, float *hc, float *m, float *n, float *u0, float *v0,
                                              float *w0, void *stream)
{
  if (!grid || grid->Nx < 3 || grid->Ny < 3 || grid->Nz < 2 || !(grid->dx > 0) || !(grid->dy > 0) ||
      !grid->dz_array || n_buildings < 0 || (n_buildings > 0 && !b) || !in || !icellflag || !e || !f || !g ||
      !hc || !m || !n || !u0 || !v0 || !w0)
    return qesb_fail(QESB_ERR_ARG, "qesb_city_build_device: bad arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  CityGrid G;
  G.nx = grid->Nx + 1;
  G.ny = grid->Ny + 1;
  G.nz = grid->Nz + 2;
  G.X = grid->Nx;
  G.XY = (long)grid->Nx * grid->Ny;
  G.FX = grid->Nx + 1;
  G.FXY = (long)(grid->Nx + 1) * (grid->Ny + 1);
  const float dx = grid->dx, dy = grid->dy;
  const float *dz = grid->dz_array;

  // host side: vertical grid, building boxes, profile (as qesb_city_build)
  std::vector<float> zf(G.nz, 0.0f), z(G.nz - 1, 0.0f);
  zf[0] = -dz[0];
  zf[1] = 0.0f;
  for (int k = 2; k < G.nz; ++k) zf[k] = zf[k - 1] + dz[k - 1];
  z[0] = -0.5f * dz[0];
  for (int k = 1; k < G.nz - 1; ++k) z[k] = 0.5f * (zf[k] + zf[k + 1]);
  std::vector<DevBuilding> bl(std::max(n_buildings, 1));
  for (int q = 0; q < n_buildings; ++q) {
    DevBuilding &d = bl[q];
    const float xs = b[q].x_start, ys = b[q].y_start;
    d.px[0] = d.px[4] = xs;
    d.py[0] = d.py[4] = ys;
    d.px[1] = xs - b[q].width * 0.0f;
    d.py[1] = ys + b[q].width * 1.0f;
    d.px[2] = d.px[1] + b[q].length * 1.0f;
    d.py[2] = d.py[1] + b[q].length * 0.0f;
    d.px[3] = xs + b[q].length * 1.0f;
    d.py[3] = ys + b[q].length * 0.0f;
    float x_min = d.px[0], x_max = d.px[0], y_min = d.py[0], y_max = d.py[0];
    for (int v = 1; v < 5; ++v) {
      x_max = std::max(x_max, d.px[v]);
      x_min = std::min(x_min, d.px[v]);
      y_max = std::max(y_max, d.py[v]);
      y_min = std::min(y_min, d.py[v]);
    }
    d.i_start = (int)(x_min / dx);
    d.i_end = (int)((x_max / dx) + 1);
    d.j_start = (int)(y_min / dy);
    d.j_end = (int)((y_max / dy) + 1);
    const float height_eff = b[q].height + b[q].base_height;
    d.k_start = 1;
    d.k_end = 1;
    for (int k = 1; k < (int)z.size(); ++k) {
      d.k_start = k;
      if (b[q].base_height <= zf[k + 1]) break;
    }
    for (int k = 0; k < (int)z.size(); ++k) {
      d.k_end = k + 1;
      if (height_eff < z[k + 1]) break;
    }
  }
  std::vector<float> tab(3 * G.nz, 0.0f);  // up[nz], vp[nz], dz[nz]
  const float theta = (float)((270.0 - in->dir_deg) * M_PI / 180.0);
  for (int k = 1; k < G.nz - 1; ++k) {
    const float sc = std::pow((z[k] - 0.0f) / in->z_ref, in->p);
    tab[k] = std::cos(theta) * in->u_ref * sc;
    tab[G.nz + k] = std::sin(theta) * in->u_ref * sc;
  }
  for (int k = 0; k < G.nz - 1; ++k) tab[2 * G.nz + k] = dz[k];

  // upload the building list and tables (one stream-ordered allocation)
  const size_t bbytes = sizeof(DevBuilding) * bl.size(), tbytes = sizeof(float) * tab.size();
  unsigned char *scratch = nullptr;
  CK(cudaMallocAsync((void **)&scratch, bbytes + tbytes, s));
  DevBuilding *d_bld = reinterpret_cast<DevBuilding *>(scratch);
  float *d_tab = reinterpret_cast<float *>(scratch + bbytes);
  cudaError_t ce = cudaMemcpyAsync(d_bld, bl.data(), bbytes, cudaMemcpyHostToDevice, s);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(d_tab, tab.data(), tbytes, cudaMemcpyHostToDevice, s);
  if (ce == cudaSuccess) {
    const long nc = G.XY * (G.nz - 1);
    k_city_flags_init<<<(unsigned)std::min<long>((nc + 255) / 256, 148L * 16), 256, 0, s>>>(G, icellflag);
    if (n_buildings > 0) k_city_flags_bld<<<n_buildings, 256, 0, s>>>(G, dx, dy, d_bld, icellflag);
    k_city_walls<<<dim3(1, G.ny - 1, G.nz - 1), 256, 0, s>>>(G, dx, d_tab + 2 * G.nz, icellflag, e, f, g, hc, m, n);
    k_city_winds<<<dim3(1, G.ny, G.nz), 256, 0, s>>>(G, d_tab, d_tab + G.nz, icellflag, u0, v0, w0);
    ce = cudaGetLastError();
  }
  // the host vectors are locals: the copies must finish before returning
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
  cudaFreeAsync(scratch, s);
  if (ce != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "qesb_city_build_device: %s", cudaGetErrorString(ce));
  return QESB_OK;
}
