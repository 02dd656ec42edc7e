// qesb_solve_noalloc: the lambda solve without any device allocation.
//
// Some callers cannot call cudaMalloc: code whose GPU memory is wholly owned
// by another allocator (a framework's caching allocator that has reserved
// the device, a host application with a fixed device-memory budget), and
// long-running coupling loops that must not allocate or free after start-up,
// where each allocation would cost a device synchronisation and risk
// fragmentation. For them this entry point solves with scratch memory that
// the library carries itself: one file-scope device array, sized at build
// time, which every GPU that loads the library holds until the process ends.
//
// It is the full-coefficient red-black solve of qesb_solve_device in the
// reference's own layouts, operating in place on the caller's lambda, with
// the same per-operation rounding (this file is compiled with -fmad=false),
// so its results equal the handle-based entry point's bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "qesb.h"
#include "qesb_device.cuh"
#include "qesb_internal.h"

using namespace qesb;

namespace {

// Scratch layout inside the array (offsets in bytes, each 256-byte aligned):
//   [0, 256)                  SolveState
//   [256, 256 + 8*MAX_ITERS)  per-iteration FP64 max|dlambda|
//   then                      dz_array (MAX_Z floats)
//   then                      R, one float per cell (reference cell layout)
constexpr size_t kStateOff = 0;
constexpr size_t kErrOff = 256;
constexpr size_t kDzOff = kErrOff + (size_t)QESB_NOALLOC_MAX_ITERS * sizeof(double);
constexpr size_t kROff = kDzOff + (((size_t)QESB_NOALLOC_MAX_Z * sizeof(float) + 255) / 256) * 256;
static_assert(sizeof(SolveState) <= 256, "state slot too small");
static_assert(kROff < QESB_NOALLOC_SCRATCH_BYTES, "scratch too small for its fixed parts");

}  // namespace

// The scratch array. In host code this name is only a stand-in for the
// symbol; its device address comes from cudaGetSymbolAddress (below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[QESB_NOALLOC_SCRATCH_BYTES];

namespace {

struct NaGrid {
  int X, Y, Z;          // cells: nx-1, ny-1, nz-1
  int FX, FY, FZ;       // faces: nx, ny, nz
  long XY, FXY;
  __device__ long cell(int i, int j, int k) const { return i + (long)j * X + (long)k * XY; }
  __device__ long face(int i, int j, int k) const { return i + (long)j * FX + (long)k * FXY; }
};

// R, Solver_CPU.cpp:56-77 (same expression and promotions as k_divergence).
__global__ void k_na_divergence(NaGrid G, const float *__restrict__ e, const float *__restrict__ f,
                                const float *__restrict__ g, const float *__restrict__ h,
                                const float *__restrict__ m, const float *__restrict__ n,
                                const float *__restrict__ u0, const float *__restrict__ v0,
                                const float *__restrict__ w0, const float *__restrict__ dz, float dx,
                                float dy, float *__restrict__ R)
{
  const int j = blockIdx.y, k = blockIdx.z + 1;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x) {
    const long c = G.cell(i, j, k), fc = G.face(i, j, k);
    const float xt = (e[c] * u0[fc + 1] - f[c] * u0[fc]) * dx;
    const float yt = (g[c] * v0[fc + G.FX] - h[c] * v0[fc]) * dy;
    const double mt = (double)(m[c] * dz[k]) * 0.5 * (double)(dz[k] + dz[k + 1]) * (double)w0[fc + G.FXY];
    const float nt = n[c] * dz[k] * 0.5f * (dz[k] + dz[k - 1]) * w0[fc];
    R[c] = (float)(-2.0 * ((double)(xt + yt) + (mt - (double)nt)));
  }
}

// One colour of the red-black sweep in place on the caller's lambda
// (Solver_CPU_RB.cpp:110-151), error folded into err[it] per block.
__global__ void __launch_bounds__(128) k_na_sor(NaGrid G, int colour, float *__restrict__ L,
                                                const float *__restrict__ pe, const float *__restrict__ pf,
                                                const float *__restrict__ pg, const float *__restrict__ ph,
                                                const float *__restrict__ pm, const float *__restrict__ pn,
                                                const float *__restrict__ R, double *__restrict__ err,
                                                const SolveState *__restrict__ st)
{
  if (st->done) return;
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  const int o = (colour + 1 + j + k) & 1;
  const int i = 1 + 2 * (int)(blockIdx.x * blockDim.x + threadIdx.x) + o;
  double d = 0.0;
  if (i <= G.X - 2) {
    const long c = G.cell(i, j, k);
    const float e = pe[c], f = pf[c], g = pg[c], h = ph[c], m = pm[c], n = pn[c];
    const float old = L[c];
    const float nv = (kOmega / (e + f + g + h + m + n)) *
                         (e * L[c + 1] + f * L[c - 1] + g * L[c + G.X] + h * L[c - G.X] + m * L[c + G.XY] +
                          n * L[c - G.XY] - R[c]) +
                     (1.0f - kOmega) * old;
    L[c] = nv;
    d = fabs((double)nv - (double)old);
  }
  block_max_to(err + st->it, d);
}

__global__ void k_na_mirror(NaGrid G, float *__restrict__ L, const SolveState *__restrict__ st)
{
  if (st->done) return;
  const int j = blockIdx.y;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x) {
    const long c = G.cell(i, j, 0);
    L[c] = L[c + G.XY];
  }
}

// Loop condition `iter < itermax && max_error > tol` after each iteration.
__global__ void k_na_poll(SolveState *st, const double *__restrict__ err, double tol, int itermax)
{
  if (st->done) return;
  const int it = st->it;
  const double e = err[it];
  st->residual = e;
  st->it = it + 1;
  if (isnan(e)) {
    st->done = 1;
    st->nan = 1;
  } else if (!(e > tol)) {
    st->done = 1;
    st->converged = 1;
  } else if (it + 1 >= itermax) {
    st->done = 1;
  }
}

// Correction and solid-face zeroing, Solver_CPU.cpp:157-231 (as k_correct).
__global__ void k_na_correct(NaGrid G, const float *__restrict__ L, const float *__restrict__ f,
                             const float *__restrict__ h, const float *__restrict__ n,
                             const int *__restrict__ flag, const float *__restrict__ u0,
                             const float *__restrict__ v0, const float *__restrict__ w0,
                             const float *__restrict__ dz, float dx, float dy, float *__restrict__ u,
                             float *__restrict__ v, float *__restrict__ w)
{
  const int j = blockIdx.y, k = blockIdx.z;
  const float half = 1.0f / (2.0f * 1.0f);
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.FX; i += gridDim.x * blockDim.x) {
    const long q = G.face(i, j, k);
    float uu = u0[q], vv = v0[q], ww = w0[q];
    if (i >= 1 && i <= G.FX - 2 && j >= 1 && j <= G.FY - 2 && k >= 1 && k <= G.FZ - 3) {
      const long c = G.cell(i, j, k);
      const float lc = L[c];
      uu = u0[q] + half * f[c] * dx * (lc - L[c - 1]);
      vv = v0[q] + half * h[c] * dy * (lc - L[c - G.X]);
      ww = w0[q] + half * n[c] * dz[k] * (lc - L[c - G.XY]);
    }
    const bool kin = k >= 1 && k <= G.FZ - 2;
    const bool ic = i <= G.X - 1, jc = j <= G.Y - 1;
    if (kin && jc && ((ic && is_solid(flag[G.cell(i, j, k)])) || (i >= 1 && is_solid(flag[G.cell(i - 1, j, k)]))))
      uu = 0.0f;
    if (kin && ic && ((jc && is_solid(flag[G.cell(i, j, k)])) || (j >= 1 && is_solid(flag[G.cell(i, j - 1, k)]))))
      vv = 0.0f;
    if (ic && jc && ((kin && is_solid(flag[G.cell(i, j, k)])) ||
                     (k - 1 >= 1 && k - 1 <= G.FZ - 2 && is_solid(flag[G.cell(i, j, k - 1)]))))
      ww = 0.0f;
    u[q] = uu;
    v[q] = vv;
    w[q] = ww;
  }
}

// Device address of the scratch array, looked up once per device and kept
// for the process. cudaDeviceReset destroys the context that holds the
// array; a later context may place it elsewhere, so a process that resets a
// device must not call this entry point on that device again.
std::mutex g_na_mu;
unsigned char *g_na_addr[64] = {};

qesb_status scratch_address(unsigned char **out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "qesb_solve_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return qesb_fail(QESB_ERR_NODEV, "qesb_solve_noalloc: device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return qesb_fail(QESB_ERR_CUDA, "qesb_solve_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_na_addr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_na_addr[dev];
  return QESB_OK;
}

#define NA_CK(call)                                                                                \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return qesb_fail(QESB_ERR_CUDA, "qesb_solve_noalloc: %s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

}  // namespace

extern "C" qesb_status qesb_solve_noalloc(const qesb_grid *grid, float tol, int itermax, const float *e,
                                          const float *f, const float *g, const float *hc, const float *m,
                                          const float *n, const int *icellflag, const float *u0,
                                          const float *v0, const float *w0, float *lambda, float *u, float *v,
                                          float *w, void *stream, qesb_stats *st)
{
  if (!grid || grid->Nx < 3 || grid->Ny < 3 || grid->Nz < 2 || !(grid->dx > 0) || !(grid->dy > 0) ||
      !grid->dz_array)
    return qesb_fail(QESB_ERR_ARG, "qesb_solve_noalloc: grid needs Nx, Ny >= 3, Nz >= 2, dx, dy > 0 and dz_array");
  if (!e || !f || !g || !hc || !m || !n || !icellflag || !u0 || !v0 || !w0 || !lambda || !u || !v || !w)
    return qesb_fail(QESB_ERR_ARG, "qesb_solve_noalloc: null array");
  // launch grids put the rows (Ny, or Ny + 1 faces) in grid.y, whose limit is 65535
  if (grid->Ny + 1 > 65535)
    return qesb_fail(QESB_ERR_ARG, "qesb_solve_noalloc: Ny = %d exceeds the limit of 65534 rows", grid->Ny);
  if (itermax < 0 || itermax > QESB_NOALLOC_MAX_ITERS)
    return qesb_fail(QESB_ERR_ARG, "qesb_solve_noalloc: itermax %d outside [0, %d]", itermax, QESB_NOALLOC_MAX_ITERS);
  const long ncell = (long)grid->Nx * grid->Ny * (grid->Nz + 1);
  if (grid->Nz + 1 > QESB_NOALLOC_MAX_Z || ncell > QESB_NOALLOC_MAX_CELLS)
    return qesb_fail(QESB_ERR_ARG,
                     "qesb_solve_noalloc: grid of %ld cells (%d layers) exceeds the built-in scratch "
                     "(at most %ld cells and %d layers); use qesb_create/qesb_solve_device",
                     ncell, grid->Nz + 1, (long)QESB_NOALLOC_MAX_CELLS, QESB_NOALLOC_MAX_Z);
  NaGrid G;
  G.X = grid->Nx;
  G.Y = grid->Ny;
  G.Z = grid->Nz + 1;
  G.FX = grid->Nx + 1;
  G.FY = grid->Ny + 1;
  G.FZ = grid->Nz + 2;
  G.XY = (long)G.X * G.Y;
  G.FXY = (long)G.FX * G.FY;

  unsigned char *base = nullptr;
  qesb_status s0 = scratch_address(&base);
  if (s0 != QESB_OK) return s0;
  SolveState *d_state = reinterpret_cast<SolveState *>(base + kStateOff);
  double *d_err = reinterpret_cast<double *>(base + kErrOff);
  float *d_dz = reinterpret_cast<float *>(base + kDzOff);
  float *d_R = reinterpret_cast<float *>(base + kROff);
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  // the array keeps the previous call's contents: reset what must start at zero
  NA_CK(cudaMemsetAsync(d_state, 0, sizeof(SolveState), s));
  NA_CK(cudaMemsetAsync(d_err, 0, sizeof(double) * std::max(itermax, 1), s));
  NA_CK(cudaMemcpyAsync(d_dz, grid->dz_array, sizeof(float) * G.Z, cudaMemcpyHostToDevice, s));

  const dim3 rows((G.X + 255) / 256, G.Y, G.Z - 2);
  k_na_divergence<<<rows, 256, 0, s>>>(G, e, f, g, hc, m, n, u0, v0, w0, d_dz, grid->dx, grid->dy, d_R);
  NA_CK(cudaGetLastError());
  int launches = 1;
  SolveState hst{};
  if (itermax > 0) {
    const int nthr = 128;
    const dim3 sgrid(((G.X - 2) / 2 + 1 + nthr - 1) / nthr, G.Y - 2, G.Z - 2);
    const dim3 mgrid((G.X + 255) / 256, G.Y, 1);
    const int chunk = 64;
    for (int base_it = 0; base_it < itermax; base_it += chunk) {
      const int cnt = std::min(chunk, itermax - base_it);
      for (int t = 0; t < cnt; ++t) {
        for (int colour = 0; colour < 2; ++colour)
          k_na_sor<<<sgrid, nthr, 0, s>>>(G, colour, lambda, e, f, g, hc, m, n, d_R, d_err, d_state);
        k_na_mirror<<<mgrid, 256, 0, s>>>(G, lambda, d_state);
        k_na_poll<<<1, 1, 0, s>>>(d_state, d_err, (double)tol, itermax);
      }
      launches += 4 * cnt;
      NA_CK(cudaGetLastError());
      NA_CK(cudaMemcpyAsync(&hst, d_state, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
      NA_CK(cudaStreamSynchronize(s));
      if (hst.done) break;
    }
  }
  const dim3 faces((G.FX + 255) / 256, G.FY, G.FZ);
  k_na_correct<<<faces, 256, 0, s>>>(G, lambda, f, hc, n, icellflag, u0, v0, w0, d_dz, grid->dx, grid->dy, u, v, w);
  NA_CK(cudaGetLastError());
  ++launches;
  NA_CK(cudaStreamSynchronize(s));
  if (st) {
    st->iterations = itermax > 0 ? hst.it : 0;
    st->converged = hst.converged;
    st->residual = itermax > 0 ? hst.residual : 1.0;
    st->ms_total = 0.0;
    st->ms_sor = 0.0;
    st->path = 0;
    st->sweeps_per_launch = 1;
    st->launches = launches;
    st->pre_iterations = 0;
    st->max_divergence = -1.0;
    st->window_drift = -1.0;
    st->ms_sweeps = -1.0;
  }
  if (hst.nan) return qesb_fail(QESB_ERR_NUMERIC, "qesb_solve_noalloc: NaN in lambda (iteration %d)", hst.it);
  return QESB_OK;
}
