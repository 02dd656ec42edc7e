// B200-native QES-Winds lambda solve: device kernels and the C ABI of
// include/qesb.h.
//
// Reference path replaced: Solver::solve (src/winds/Solver_CPU.cpp:42-238,
// Solver_CPU_RB.cpp:41-291), created through SolverFactory::create
// (src/winds/SolverFactory.cpp:35-60).
//
// This translation unit is compiled with -fmad=false: every float and double
// operation below rounds on its own, as the reference's host code does when
// built without FMA contraction. With that, the red-black sweep reproduces
// Solver_CPU_RB bit for bit (same per-cell expression, same colour order),
// R reproduces Solver_CPU.cpp:64-74 bit for bit, and the correction
// reproduces Solver_CPU.cpp:157-231 bit for bit.
//
// Device layout (per handle). Cell fields that the sweep touches (lambda,
// R, the wall mask, the full coefficients) live in a padded layout:
//   index(i, j, k) = k*PLANE + (j + GY)*PX + (i + GX),  PLANE = PX*PY,
//   PX = roundup(X + 2*GX, 32) (rows start on 128-byte boundaries),
//   PY = Y + 2*GY, X = nx-1, Y = ny-1, k in [0, nz-2].
// The guard cells are zero and never updated; they let tiled kernels read a
// halo beyond the domain edge without bounds checks. Inputs and outputs in
// the reference layouts (cells i + j*X + k*X*Y, faces i + j*nx + k*nx*ny)
// stay as the caller gave them.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "qesb.h"
#include "qesb_internal.h"
#include "qesb_device.cuh"
#include "qesb_sor_tiled.cuh"
#include "qesb_sor_split.cuh"
#include "qesb_sor_zm.cuh"
#include "qesb_wall_log.cuh"
#include "qesb_fp64.cuh"
#include "qesb_sor_bulk.cuh"

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

qesb_status qesb_fail(qesb_status s, const char *fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return qesb_fail(e_ == cudaErrorMemoryAllocation ? QESB_ERR_NOMEM : QESB_ERR_CUDA,           \
                       "%s failed at %s:%d: %s", #call, __FILE__, __LINE__, cudaGetErrorString(e_)); \
  } while (0)

#define CKS(expr)                                                                                  \
  do {                                                                                             \
    qesb_status s_ = (expr);                                                                       \
    if (s_ != QESB_OK) return s_;                                                                  \
  } while (0)

using namespace qesb;

// ---------------------------------------------------------------------------
// kernels: set-up
// ---------------------------------------------------------------------------

// Per-layer coefficient values: for each of the six coefficients and each
// updated layer k, the largest value over the updated cells. With stair-step
// walls every value is either 0 or this one value.
__global__ void k_layer_max(DevGrid G, const float *__restrict__ e, const float *__restrict__ f,
                            const float *__restrict__ g, const float *__restrict__ h,
                            const float *__restrict__ m, const float *__restrict__ n,
                            unsigned *__restrict__ vmax, int *__restrict__ bad)
{
  // one block per 8 updated rows j of layer k, threads along x; one atomic per block and coefficient
  const int k = blockIdx.y + 1, j0 = 1 + blockIdx.x * 8;
  const float *cf[6] = {e, f, g, h, m, n};
  float mx[6] = {0, 0, 0, 0, 0, 0};
  bool b = false;
  for (int j = j0; j < min(j0 + 8, G.Y - 1); ++j)
    for (int i = 1 + threadIdx.x; i <= G.X - 2; i += blockDim.x) {
      const long c = G.cell(i, j, k);
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const float v = cf[q][c];
        b |= !(v >= 0.0f) || isinf(v);  // negative, NaN or Inf: no packing
        mx[q] = fmaxf(mx[q], v);
      }
    }
  if (__syncthreads_or(b) && threadIdx.x == 0) atomicExch(bad, 1);
  __shared__ float red[6][8];
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const float v = warp_max_f(mx[q]);
    if ((threadIdx.x & 31) == 0) red[q][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    float v = 0.0f;
    for (int q = 0; q < nw; ++q) v = fmaxf(v, red[threadIdx.x][q]);
    atomicMax(&vmax[threadIdx.x * G.Z + k], __float_as_uint(v));
  }
}

// Builds the 6-bit wall mask (bit q set when coefficient q is non-zero) and
// flags any value that is neither 0 nor its layer's value. One block per
// updated (row j, layer k), threads along x.
__global__ void k_build_mask(DevGrid G, const float *__restrict__ e, const float *__restrict__ f,
                             const float *__restrict__ g, const float *__restrict__ h,
                             const float *__restrict__ m, const float *__restrict__ n,
                             const unsigned *__restrict__ vmax, uint8_t *__restrict__ mask,
                             int *__restrict__ bad)
{
  const int j = blockIdx.x + 1, k = blockIdx.y + 1;
  const float *cf[6] = {e, f, g, h, m, n};
  float ref[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) ref[q] = __uint_as_float(vmax[q * G.Z + k]);
  bool b = false;
  for (int i = 1 + threadIdx.x; i <= G.X - 2; i += blockDim.x) {
    const long c = G.cell(i, j, k);
    unsigned bits = 0;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const float v = cf[q][c];
      if (v == ref[q] && v != 0.0f) bits |= 1u << q;
      else if (v != 0.0f) b = true;
    }
    mask[G.pad(i, j, k)] = (uint8_t)bits;
  }
  if (__syncthreads_or(b) && threadIdx.x == 0) atomicExch(bad, 1);
}

// inv[k*64 + bits] = omega / (e + f + g + h + m + n) with absent terms 0,
// summed in the reference's order (Solver_CPU.cpp:107).
__global__ void k_inv_table(DevGrid G, const unsigned *__restrict__ vmax, float *__restrict__ inv,
                            float *__restrict__ val, float omega)
{
  const int k = blockIdx.x, bits = threadIdx.x;
  float v[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) v[q] = __uint_as_float(vmax[q * G.Z + k]);
  float s = (bits & 1 ? v[0] : 0.0f);
  s = s + (bits & 2 ? v[1] : 0.0f);
  s = s + (bits & 4 ? v[2] : 0.0f);
  s = s + (bits & 8 ? v[3] : 0.0f);
  s = s + (bits & 16 ? v[4] : 0.0f);
  s = s + (bits & 32 ? v[5] : 0.0f);
  inv[k * 64 + bits] = omega / s;
  if (bits < 6) val[bits * G.Z + k] = v[bits];
}

// Natural -> padded copy of the six coefficients (full-coefficient path).
__global__ void k_pad_coefs(DevGrid G, const float *__restrict__ e, const float *__restrict__ f,
                            const float *__restrict__ g, const float *__restrict__ h,
                            const float *__restrict__ m, const float *__restrict__ n,
                            float *__restrict__ pe, float *__restrict__ pf, float *__restrict__ pg,
                            float *__restrict__ ph, float *__restrict__ pm, float *__restrict__ pn)
{
  const int j = blockIdx.y, k = blockIdx.z;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x) {
    const long c = G.cell(i, j, k), p = G.pad(i, j, k);
    pe[p] = e[c];
    pf[p] = f[c];
    pg[p] = g[c];
    ph[p] = h[c];
    pm[p] = m[c];
    pn[p] = n[c];
  }
}

// Divergence of the initial field, Solver_CPU.cpp:56-77, into padded R.
// The reference expression mixes precisions: (-2.0f * pow(alpha1, 2.0)) and
// the m-term's 0.5 literal are double; the x, y and n terms are float.
__global__ void k_divergence(DevGrid G, const float *__restrict__ e, const float *__restrict__ f,
                             const float *__restrict__ g, const float *__restrict__ h,
                             const float *__restrict__ m, const float *__restrict__ n,
                             const float *__restrict__ u0, const float *__restrict__ v0,
                             const float *__restrict__ w0, const float *__restrict__ dz,
                             float dx, float dy, float *__restrict__ R)
{
  const int j = blockIdx.y, k = blockIdx.z + 1;  // k in [1, nz-3]
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x) {
    const long c = G.cell(i, j, k), fc = G.face(i, j, k);
    const float xt = (e[c] * u0[fc + 1] - f[c] * u0[fc]) * dx;
    const float yt = (g[c] * v0[fc + G.FX] - h[c] * v0[fc]) * dy;
    const double mt = (double)(m[c] * dz[k]) * 0.5 * (double)(dz[k] + dz[k + 1]) * (double)w0[fc + G.FXY];
    const float nt = n[c] * dz[k] * 0.5f * (dz[k] + dz[k - 1]) * w0[fc];
    R[G.pad(i, j, k)] = (float)(-2.0 * ((double)(xt + yt) + (mt - (double)nt)));
  }
}

// The same from the packed wall mask: on the updated cells every coefficient
// is exactly 0 or its layer's value (the packed path's precondition), so
// reading the 1-byte mask instead of the six arrays gives the same R bit for
// bit; the boundary cells, which have no mask, read the arrays.
__global__ void k_divergence_packed(DevGrid G, const uint8_t *__restrict__ mask, const float *__restrict__ val,
                                    const float *__restrict__ e, const float *__restrict__ f,
                                    const float *__restrict__ g, const float *__restrict__ h,
                                    const float *__restrict__ m, const float *__restrict__ n,
                                    const float *__restrict__ u0, const float *__restrict__ v0,
                                    const float *__restrict__ w0, const float *__restrict__ dz,
                                    float dx, float dy, float *__restrict__ R)
{
  const int j = blockIdx.y, k = blockIdx.z + 1;  // k in [1, nz-3]
  const bool row_in = j >= 1 && j <= G.Y - 2;
  float lv[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) lv[q] = __ldg(val + q * G.Z + k);
  const float dzk = dz[k], dzp = dz[k + 1], dzm = dz[k - 1];
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x) {
    const long c = G.cell(i, j, k), fc = G.face(i, j, k);
    float ce, cf, cg, ch, cm, cn;
    if (row_in && i >= 1 && i <= G.X - 2) {
      const unsigned mb = mask[G.pad(i, j, k)];
      ce = mb & 1u ? lv[0] : 0.0f;
      cf = mb & 2u ? lv[1] : 0.0f;
      cg = mb & 4u ? lv[2] : 0.0f;
      ch = mb & 8u ? lv[3] : 0.0f;
      cm = mb & 16u ? lv[4] : 0.0f;
      cn = mb & 32u ? lv[5] : 0.0f;
    } else {
      ce = e[c], cf = f[c], cg = g[c], ch = h[c], cm = m[c], cn = n[c];
    }
    const float xt = (ce * u0[fc + 1] - cf * u0[fc]) * dx;
    const float yt = (cg * v0[fc + G.FX] - ch * v0[fc]) * dy;
    const double mt = (double)(cm * dzk) * 0.5 * (double)(dzk + dzp) * (double)w0[fc + G.FXY];
    const float nt = cn * dzk * 0.5f * (dzk + dzm) * w0[fc];
    R[G.pad(i, j, k)] = (float)(-2.0 * ((double)(xt + yt) + (mt - (double)nt)));
  }
}

// Natural <-> padded lambda.
__global__ void k_lambda_to_pad(DevGrid G, const float *__restrict__ src, float *__restrict__ dst)
{
  const int j = blockIdx.y, k = blockIdx.z;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x)
    dst[G.pad(i, j, k)] = src[G.cell(i, j, k)];
}
__global__ void k_lambda_from_pad(DevGrid G, const float *__restrict__ src, float *__restrict__ dst)
{
  const int j = blockIdx.y, k = blockIdx.z;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x)
    dst[G.cell(i, j, k)] = src[G.pad(i, j, k)];
}

// ---------------------------------------------------------------------------
// kernels: iteration (full-coefficient path, one colour per launch)
// ---------------------------------------------------------------------------

// One colour of the red-black sweep (Solver_CPU_RB.cpp:110-151): cells with
// (i + j + k) % 2 == colour in i in [1, nx-3], j in [1, ny-3], k in [1, nz-3].
// The per-iteration error max|lambda_new - lambda_old| is formed in double
// at update time (each cell changes once per iteration) and folded into
// err[it] with one 64-bit atomicMax per block.
__global__ void __launch_bounds__(128) k_sor_full(DevGrid G, int colour, float *__restrict__ L,
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
    const long p = G.pad(i, j, k);
    const float e = pe[p], f = pf[p], g = pg[p], h = ph[p], m = pm[p], n = pn[p];
    const float old = L[p];
    const float nv = (kOmega / (e + f + g + h + m + n)) *
                         (e * L[p + 1] + f * L[p - 1] + g * L[p + G.PX] + h * L[p - G.PX] +
                          m * L[p + G.PLANE] + n * L[p - G.PLANE] - R[p]) +
                     (1.0f - kOmega) * old;
    L[p] = nv;
    d = fabs((double)nv - (double)old);
  }
  block_max_to(err + st->it, d);
}

// Ground mirror lambda(k=0) <- lambda(k=1) over the whole plane (Solver_CPU.cpp:119-126).
__global__ void k_mirror(DevGrid G, float *__restrict__ L, const SolveState *__restrict__ st)
{
  if (st->done) return;
  const int j = blockIdx.y;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x) {
    const long p = G.pad(i, j, 0);
    L[p] = L[p + G.PLANE];
  }
}

// Convergence poll after a launch of up to kmax iterations starting at
// st->it: the reference loop condition `iter < itermax && max_error > tol`
// (Solver_CPU.cpp:93) checked for each of the launch's iterations in order,
// with max_error in double. If the stop falls inside a fused launch, that
// launch ran past it; the poll records how many of its iterations count so
// the host re-runs exactly those from the launch's input buffer. A NaN error
// stops the solve and is reported. `parity` is the launch's output buffer.
__global__ void k_poll(SolveState *st, const double *__restrict__ err, double tol, int itermax,
                       int kmax, int parity)
{
  if (st->done) return;
  const int t0 = st->it;
  const int nit = min(kmax, itermax - t0);
  st->cur = parity;
  for (int t = 0; t < nit; ++t) {
    const double e = err[t0 + t];
    st->residual = e;
    const bool nan = isnan(e);
    if (nan || !(e > tol)) {
      st->done = 1;
      st->nan = nan;
      st->converged = !nan;
      st->it = t0 + t + 1;
      if (t + 1 < nit && !nan) {
        st->redo = t + 1;
        st->redo_t0 = t0;
        st->redo_par = parity;
      }
      return;
    }
  }
  st->it = t0 + nit;
  if (st->it >= itermax) st->done = 1;
}

// Window rule on the full-coefficient path (one domain, padded layout):
// max|lambda - snapshot| over the n4 float4 of the layout into st->wacc,
// FP64 exact, and the snapshot takes lambda's values; skipped once the loop
// has stopped. k_window_poll_full then applies the rule.
__global__ void k_window_full(const float4 *__restrict__ L, float4 *__restrict__ S, long n4, SolveState *st)
{
  if (st->done) return;
  double dmax = 0.0;
  for (long i = threadIdx.x + (long)blockIdx.x * blockDim.x; i < n4; i += (long)gridDim.x * blockDim.x) {
    const float4 a = L[i], o = S[i];
    const double d[4] = {fabs((double)a.x - (double)o.x), fabs((double)a.y - (double)o.y),
                         fabs((double)a.z - (double)o.z), fabs((double)a.w - (double)o.w)};
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (d[q] > dmax || d[q] != d[q]) dmax = d[q];
    S[i] = a;
  }
  block_max_to(&st->wacc, dmax);
}

__global__ void k_window_poll_full(SolveState *st, double wtol)
{
  if (st->done) return;
  const double d = st->wacc;
  st->wacc = 0.0;
  st->wdrift = d;
  if (isnan(d)) {
    st->done = 1;
    st->nan = 1;
  } else if (d <= wtol) {
    st->done = 1;
    st->converged = 2;
  }
}

// Final divergence check in FP64: max over fluid cells (icellflag == 1),
// i in [1, nx-3], j in [1, ny-3], k in [1, kmax], of
//   |(u[i+1]-u[i])/dx + (v[j+1]-v[j])/dy + (w[k+1]-w[k])/dz[k]|
// evaluated in double. kmax = nz-4 leaves out the last solved layer, whose top
// face the reference never corrects (Solver_CPU.cpp:197-209 stops at k = nz-3).
__global__ void k_max_divergence(DevGrid G, const int *__restrict__ flag, const float *__restrict__ u,
                                 const float *__restrict__ v, const float *__restrict__ w,
                                 const float *__restrict__ dz, float dx, float dy, int kmax, double *out)
{
  // a warp per row j of layer k (eight rows per block), lanes along x; one atomic per block
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z + 1;
  double mx = 0.0;
  if (j <= G.Y - 2 && k <= kmax) {
    for (int i = 1 + threadIdx.x; i <= G.X - 2; i += blockDim.x) {
      if (flag[G.cell(i, j, k)] != 1) continue;
      const long fc = G.face(i, j, k);
      const double d = ((double)u[fc + 1] - u[fc]) / dx + ((double)v[fc + G.FX] - v[fc]) / dy +
                       ((double)w[fc + G.FXY] - w[fc]) / dz[k];
      const double a = fabs(d);
      if (a > mx || a != a) mx = a;
    }
  }
  block_max_to(out, mx);
}

// ---------------------------------------------------------------------------
// kernels: velocity correction (Solver_CPU.cpp:157-231)
// ---------------------------------------------------------------------------
// One thread per face (i, j, k). Each face's final value is: 0 if it is a
// face of a solid cell (icellflag 0 or 2) with k in [1, nz-2] — the zeroing
// pass runs last in the reference, so it wins — else u0 plus the correction
// when (i, j, k) is in i in [1, nx-2], j in [1, ny-2], k in [1, nz-3], else u0.
// Gathering per face avoids the overlapping scattered writes of the
// reference's zeroing loop and gives the same result.
__global__ void k_correct(DevGrid G, const float *__restrict__ L, const float *__restrict__ f,
                          const float *__restrict__ h, const float *__restrict__ n,
                          const int *__restrict__ flag, const float *__restrict__ u0,
                          const float *__restrict__ v0, const float *__restrict__ w0,
                          const float *__restrict__ dz, float dx, float dy, float *__restrict__ u,
                          float *__restrict__ v, float *__restrict__ w)
{
  // a warp per face row (j, k), 32 faces per step along x
  const int j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
  if (j >= G.FY) return;
  const float half = 1.0f / (2.0f * 1.0f);
  for (int i = threadIdx.x; i < G.FX; i += blockDim.x) {
    const long q = G.face(i, j, k);
    float uu = u0[q], vv = v0[q], ww = w0[q];
    const bool corr = i >= 1 && i <= G.FX - 2 && j >= 1 && j <= G.FY - 2 && k >= 1 && k <= G.FZ - 3;
    if (corr) {
      const long c = G.cell(i, j, k), p = G.pad(i, j, k);
      const float lc = L[p];
      uu = u0[q] + half * f[c] * dx * (lc - L[p - 1]);
      vv = v0[q] + half * h[c] * dy * (lc - L[p - G.PX]);
      ww = w0[q] + half * n[c] * dz[k] * (lc - L[p - G.PLANE]);
    }
    const bool kin = k >= 1 && k <= G.FZ - 2;          // zeroing covers cells k in [1, nz-2]
    const bool ic = i <= G.X - 1, jc = j <= G.Y - 1;   // a cell (i, j, k) exists
    if (kin && jc && ((ic && is_solid(flag[G.cell(i, j, k)])) || (i >= 1 && is_solid(flag[G.cell(i - 1, j, k)]))))
      uu = 0.0f;
    if (kin && ic && ((jc && is_solid(flag[G.cell(i, j, k)])) || (j >= 1 && is_solid(flag[G.cell(i, j - 1, k)]))))
      vv = 0.0f;
    if (ic && jc && ((kin && is_solid(flag[G.cell(i, j, k)])) ||
                     (k - 1 >= 1 && k - 1 <= G.FZ - 2 && is_solid(flag[G.cell(i, j, k - 1)]))))
      ww = 0.0f;
    if (u) u[q] = uu;
    if (v) v[q] = vv;
    if (w) w[q] = ww;
  }
}

// ---------------------------------------------------------------------------
// kernels: warm-start network input / target / output
// ---------------------------------------------------------------------------
// The network sees planes k in [0, Dn) (Dn = nz-2: every plane but the top
// boundary) of the X x Y cell grid, channels-last [Dn][Y][X][C] BF16:
//   0: R / s  (s = max |R| over updated cells)     1: solid (icellflag 0 or 2)
//   2: dz[k] / mean(dz)                              3: boundary (cell never updated)
//   4: height of the cell centre / domain height     5..C-1: 0
__global__ void k_absmax_R(DevGrid G, const float *__restrict__ R, unsigned *__restrict__ out)
{
  // one block per 8 updated rows j of layer k, threads along x; one atomic per block
  const int k = blockIdx.y + 1, j0 = 1 + blockIdx.x * 8;
  float mx = 0.0f;
  for (int j = j0; j < min(j0 + 8, G.Y - 1); ++j)
    for (int i = 1 + threadIdx.x; i <= G.X - 2; i += blockDim.x) mx = fmaxf(mx, fabsf(R[G.pad(i, j, k)]));
  __shared__ float red[8];
  mx = warp_max_f(mx);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) mx = fmaxf(mx, red[q]);
    atomicMax(out, __float_as_uint(mx));
  }
}

__device__ __forceinline__ uint32_t bf16_bits_rne(float f)
{
  const uint32_t b = __float_as_uint(f);
  return (b + 0x7FFFu + ((b >> 16) & 1u)) >> 16;  // round to nearest even
}

// One block per (row j, layer k) of the net grid, threads along x; channels
// 0..4 as above, 5..C-1 zero, written 8 channels (16 bytes) at a time.
__global__ void k_warm_input(DevGrid G, int Dn, int C, const float *__restrict__ R, const int *__restrict__ flag,
                             const float *__restrict__ dz, const unsigned *__restrict__ smax, float dz_mean,
                             float height, uint16_t *__restrict__ x)
{
  const int j = blockIdx.y, k = blockIdx.z;
  __shared__ float s_zc;
  if (threadIdx.x == 0) {
    float zc = 0.0f;
    for (int q = 1; q < k; ++q) zc += dz[q];
    s_zc = zc + 0.5f * dz[k];
  }
  __syncthreads();
  const float inv_s = 1.0f / fmaxf(__uint_as_float(*smax), 1e-30f);
  const float c2 = dz[k] / dz_mean, c4 = s_zc / height;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G.X; i += gridDim.x * blockDim.x) {
    const bool upd = i >= 1 && i <= G.X - 2 && j >= 1 && j <= G.Y - 2 && k >= 1 && k <= G.Z - 2;
    const float ch0 = upd ? R[G.pad(i, j, k)] * inv_s : 0.0f;
    const float ch1 = is_solid(flag[G.cell(i, j, k)]) ? 1.0f : 0.0f;
    const float ch3 = upd ? 0.0f : 1.0f;
    uint4 lo;
    lo.x = bf16_bits_rne(ch0) | (bf16_bits_rne(ch1) << 16);
    lo.y = bf16_bits_rne(c2) | (bf16_bits_rne(ch3) << 16);
    lo.z = bf16_bits_rne(c4);
    lo.w = 0u;
    uint4 *dst = reinterpret_cast<uint4 *>(x + (((long)k * G.Y + j) * G.X + i) * C);
    dst[0] = lo;
    for (int q = 1; q < C / 8; ++q) dst[q] = make_uint4(0, 0, 0, 0);
  }
}

// The network input at half resolution in one pass: each voxel (xx, yy, zz)
// of the (Dn/2) x (Y/2) x (X/2) grid is the 2x2x2 average of k_warm_input's
// features of cells (2xx + a, 2yy + b, 2zz + c), each first rounded to BF16
// and summed in FP32 in k_pool2's order, then scaled by 1/8 and rounded: the
// bits of k_warm_input followed by the pooling, without the full-resolution
// tensor. One block per half-resolution (row, layer), threads along x.
__global__ void k_warm_input_half(DevGrid G, int C, const float *__restrict__ R, const int *__restrict__ flag,
                                  const float *__restrict__ dz, const unsigned *__restrict__ smax, float dz_mean,
                                  float height, uint16_t *__restrict__ x)
{
  const int yy = blockIdx.y, zz = blockIdx.z, W2 = G.X / 2, H2 = G.Y / 2;
  __shared__ float s_zc[2];
  if (threadIdx.x < 2) {
    const int k = 2 * zz + threadIdx.x;
    float zc = 0.0f;
    for (int q = 1; q < k; ++q) zc += dz[q];
    s_zc[threadIdx.x] = zc + 0.5f * dz[k];
  }
  __syncthreads();
  const float inv_s = 1.0f / fmaxf(__uint_as_float(*smax), 1e-30f);
  auto bf = [](float v) { return __uint_as_float(bf16_bits_rne(v) << 16); };
  for (int xx = blockIdx.x * blockDim.x + threadIdx.x; xx < W2; xx += gridDim.x * blockDim.x) {
    float acc[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int c = q >> 2, k = 2 * zz + c, j = 2 * yy + ((q >> 1) & 1), i = 2 * xx + (q & 1);
      const bool upd = i >= 1 && i <= G.X - 2 && j >= 1 && j <= G.Y - 2 && k >= 1 && k <= G.Z - 2;
      acc[0] += bf(upd ? R[G.pad(i, j, k)] * inv_s : 0.0f);
      acc[1] += bf(is_solid(flag[G.cell(i, j, k)]) ? 1.0f : 0.0f);
      acc[2] += bf(dz[k] / dz_mean);
      acc[3] += bf(upd ? 0.0f : 1.0f);
      acc[4] += bf(s_zc[c] / height);
    }
    uint4 lo;
    lo.x = bf16_bits_rne(acc[0] * 0.125f) | (bf16_bits_rne(acc[1] * 0.125f) << 16);
    lo.y = bf16_bits_rne(acc[2] * 0.125f) | (bf16_bits_rne(acc[3] * 0.125f) << 16);
    lo.z = bf16_bits_rne(acc[4] * 0.125f);
    lo.w = 0u;
    uint4 *dst = reinterpret_cast<uint4 *>(x + (((long)zz * H2 + yy) * W2 + xx) * C);
    dst[0] = lo;
    for (int q = 1; q < C / 8; ++q) dst[q] = make_uint4(0, 0, 0, 0);
  }
}

// Training target lambda / s and weight (1 on updated cells) on the net grid.
__global__ void k_warm_target(DevGrid G, int Dn, const float *__restrict__ L, const unsigned *__restrict__ smax,
                              float *__restrict__ tgt, float *__restrict__ w)
{
  const float inv_s = 1.0f / fmaxf(__uint_as_float(*smax), 1e-30f);
  const long V = (long)Dn * G.Y * G.X;
  for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < V; v += (long)gridDim.x * blockDim.x) {
    const int i = (int)(v % G.X), j = (int)((v / G.X) % G.Y), k = (int)(v / ((long)G.X * G.Y));
    const bool upd = i >= 1 && i <= G.X - 2 && j >= 1 && j <= G.Y - 2 && k >= 1 && k <= G.Z - 2;
    tgt[v] = upd ? L[G.pad(i, j, k)] * inv_s : 0.0f;
    w[v] = upd ? 1.0f : 0.0f;
  }
}

// lambda <- s * prediction on updated cells, 0 on the other cells of planes
// 1..Z-1, and the ground plane mirrors plane 1 (as after a solve).
__global__ void k_warm_apply(DevGrid G, int Dn, const float *__restrict__ yhead, int N,
                             const unsigned *__restrict__ smax, float *__restrict__ L)
{
  const int j = blockIdx.y, k = blockIdx.z;
  const float s = __uint_as_float(*smax);
  const int kk = k == 0 ? 1 : k;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G.X; i += gridDim.x * blockDim.x) {
    const bool upd = i >= 1 && i <= G.X - 2 && j >= 1 && j <= G.Y - 2 && kk >= 1 && kk <= G.Z - 2 && kk < Dn;
    L[G.pad(i, j, k)] = upd ? s * yhead[(((long)kk * G.Y + j) * G.X + i) * N] : 0.0f;
  }
}

// As k_warm_apply for a network run at half resolution: yhead is the
// (Dn/2) x (Y/2) x (X/2) grid, and each fine cell takes the trilinear
// interpolation of it at its centre (coarse coordinate f/2 - 1/4 per axis,
// constant beyond the outermost coarse centres), so the start carries no
// 2-cell steps for the sweeps to smooth.
__device__ __forceinline__ void up2_axis(int f, int n2, int &a, int &b, float &t)
{
  const float c = 0.5f * (float)f - 0.25f;
  const int lo = (int)floorf(c);
  t = c - (float)lo;
  a = min(max(lo, 0), n2 - 1);
  b = min(max(lo + 1, 0), n2 - 1);
}

__global__ void k_warm_apply_up2(DevGrid G, int Dn, const float *__restrict__ yhead, int N,
                                 const unsigned *__restrict__ smax, float *__restrict__ L)
{
  const int j = blockIdx.y, k = blockIdx.z;
  const float s = __uint_as_float(*smax);
  const int kk = k == 0 ? 1 : k;
  const int D2 = Dn / 2, H2 = G.Y / 2, W2 = G.X / 2;
  int z0, z1, y0, y1;
  float tz, ty;
  up2_axis(kk, D2, z0, z1, tz);
  up2_axis(j, H2, y0, y1, ty);
  // the four coarse rows this fine row interpolates between (per block)
  const float *r00 = yhead + ((long)z0 * H2 + y0) * W2 * N, *r01 = yhead + ((long)z0 * H2 + y1) * W2 * N;
  const float *r10 = yhead + ((long)z1 * H2 + y0) * W2 * N, *r11 = yhead + ((long)z1 * H2 + y1) * W2 * N;
  const bool row_upd = j >= 1 && j <= G.Y - 2 && kk >= 1 && kk <= G.Z - 2 && kk < Dn;
  float *Lrow = L + G.pad(0, j, k);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G.X; i += gridDim.x * blockDim.x) {
    const bool upd = row_upd && i >= 1 && i <= G.X - 2;
    float v = 0.0f;
    if (upd) {
      int x0, x1;
      float tx;
      up2_axis(i, W2, x0, x1, tx);
      const int a = x0 * N, b = x1 * N;
      const float c00 = r00[a] * (1.0f - tx) + r00[b] * tx;
      const float c01 = r01[a] * (1.0f - tx) + r01[b] * tx;
      const float c10 = r10[a] * (1.0f - tx) + r10[b] * tx;
      const float c11 = r11[a] * (1.0f - tx) + r11[b] * tx;
      const float c0 = c00 * (1.0f - ty) + c01 * ty, c1 = c10 * (1.0f - ty) + c11 * ty;
      v = s * (c0 * (1.0f - tz) + c1 * tz);
    }
    Lrow[i] = v;
  }
}

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
// Small transfers on a solve's critical path (state polls, domain lists,
// snapshots) run as kernels, between device memory and mapped pinned host
// memory, not as copies: a copy waits in the copy engine's queue behind any
// large transfer running for another stream (a batch's winds on their way to
// the host, the next batch's inputs on their way in), and the solve's host
// loop would wait with it. Words of [skip_lo, skip_hi) are left as they are.
__global__ void k_words(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst, int n, int skip_lo, int skip_hi)
{
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < n; i += gridDim.x * blockDim.x)
    if (i < skip_lo || i >= skip_hi) dst[i] = src[i];
  __threadfence_system();
}

__global__ void k_copy4(const float *__restrict__ src, float *__restrict__ dst, long n)
{
  const long n4 = n / 4;
  const float4 *s4 = reinterpret_cast<const float4 *>(src);
  float4 *d4 = reinterpret_cast<float4 *>(dst);
  for (long i = threadIdx.x + blockIdx.x * (long)blockDim.x; i < n4; i += (long)gridDim.x * blockDim.x) d4[i] = s4[i];
  for (long i = 4 * n4 + threadIdx.x + blockIdx.x * (long)blockDim.x; i < n; i += (long)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// dst, src: device memory or the device alias of mapped pinned memory; bytes a multiple of 4
qesb_status copy_words(void *dst, const void *src, size_t bytes, cudaStream_t s, size_t skip_lo = 0, size_t skip_hi = 0)
{
  const int n = (int)(bytes / 4);
  k_words<<<std::max(1, std::min(148, (n + 255) / 256)), 256, 0, s>>>(
      static_cast<const uint32_t *>(src), static_cast<uint32_t *>(dst), n, (int)(skip_lo / 4), (int)(skip_hi / 4));
  CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_copy_small(void *dst, const void *src, size_t bytes, void *stream)
{
  return copy_words(dst, src, bytes, static_cast<cudaStream_t>(stream));
}

__global__ void k_zero(uint32_t *__restrict__ p, long n, bool vec)
{
  const long n4 = vec ? n / 4 : 0;
  uint4 *p4 = reinterpret_cast<uint4 *>(p);
  for (long i = threadIdx.x + blockIdx.x * (long)blockDim.x; i < n4; i += (long)gridDim.x * blockDim.x)
    p4[i] = make_uint4(0, 0, 0, 0);
  for (long i = 4 * n4 + threadIdx.x + blockIdx.x * (long)blockDim.x; i < n; i += (long)gridDim.x * blockDim.x) p[i] = 0;
}

// Zeroes `bytes` (a multiple of 4) of device memory with a kernel, like the copies above.
cudaError_t zero_async(void *p, size_t bytes, cudaStream_t s)
{
  const long n = (long)(bytes / 4);
  k_zero<<<(unsigned)std::max<long>(1, std::min<long>((n / 4 + 255) / 256, 148L * 4)), 256, 0, s>>>(
      static_cast<uint32_t *>(p), n, reinterpret_cast<uintptr_t>(p) % 16 == 0);
  return cudaGetLastError();
}

// Several small copies or zero fills (src null) in one launch, one op per grid row.
constexpr int kMaxWordOps = 32;
struct WordOps {
  const uint32_t *src[kMaxWordOps];
  uint32_t *dst[kMaxWordOps];
  int n[kMaxWordOps];
  int count;
};

__global__ void k_word_ops(WordOps ops)
{
  const int q = blockIdx.y;
  if (q >= ops.count) return;
  const uint32_t *src = ops.src[q];
  uint32_t *dst = ops.dst[q];
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < ops.n[q]; i += gridDim.x * blockDim.x)
    dst[i] = src ? src[i] : 0u;
  __threadfence_system();
}

// Collects small copies and fills (bytes multiples of 4) and launches them together on flush().
struct WordBatch {
  WordOps ops{};
  int maxn = 0;
  cudaStream_t s;
  explicit WordBatch(cudaStream_t st) : s(st) {}
  qesb_status add(void *dst, const void *src, size_t bytes)
  {
    if (ops.count == kMaxWordOps) CKS(flush());
    ops.src[ops.count] = static_cast<const uint32_t *>(src);
    ops.dst[ops.count] = static_cast<uint32_t *>(dst);
    ops.n[ops.count] = (int)(bytes / 4);
    maxn = std::max(maxn, ops.n[ops.count]);
    ++ops.count;
    return QESB_OK;
  }
  qesb_status zero(void *dst, size_t bytes) { return add(dst, nullptr, bytes); }
  qesb_status flush()
  {
    if (ops.count == 0) return QESB_OK;
    k_word_ops<<<dim3(std::max(1, std::min(148, (maxn + 255) / 256)), ops.count), 256, 0, s>>>(ops);
    ops.count = 0;
    maxn = 0;
    CK(cudaGetLastError());
    return QESB_OK;
  }
};

// device -> device copy of n floats (16-byte aligned pointers)
qesb_status copy_floats(float *dst, const float *src, long n, cudaStream_t s)
{
  k_copy4<<<148 * 4, 256, 0, s>>>(src, dst, n);
  CK(cudaGetLastError());
  return QESB_OK;
}

constexpr size_t kIoBytes = 256;  // a handle's scratch for small reads

// Pinned host memory mapped into the device's address space, and its device alias.
template <class T>
qesb_status host_mapped(T **host, T **dev, size_t bytes)
{
  *host = nullptr;
  *dev = nullptr;
  if (cudaHostAlloc((void **)host, bytes, cudaHostAllocMapped) != cudaSuccess)
    return qesb_fail(QESB_ERR_NOMEM, "cudaHostAlloc (mapped) of %zu bytes failed", bytes);
  std::memset(*host, 0, bytes);
  if (cudaHostGetDevicePointer((void **)dev, *host, 0) != cudaSuccess)
    return qesb_fail(QESB_ERR_CUDA, "cudaHostGetDevicePointer failed");
  return QESB_OK;
}

// Device-side domain list for the sweep kernels: descriptors, control
// block, active list and unit offsets in one allocation of capacity n.
struct SweepList {
  unsigned char *blk = nullptr;
  unsigned char *stage = nullptr, *stage_dev = nullptr;  // mapped pinned image of blk, written by the host
  size_t bytes = 0;
  int cap = 0;
  SweepArgs a{};
  qesb_status create(int n)
  {
    static_assert(sizeof(SweepDomain) % 4 == 0 && sizeof(SweepCtl) % 8 == 0, "word copies of the list block");
    bytes = sizeof(SweepDomain) * n + sizeof(SweepCtl) + sizeof(int) * (2 * n + 1);
    bytes = (bytes + 3) / 4 * 4;
    CK(cudaMalloc((void **)&blk, bytes));
    CKS(host_mapped(&stage, &stage_dev, bytes));
    cap = n;
    a.dom = reinterpret_cast<SweepDomain *>(blk);
    a.ctl = reinterpret_cast<SweepCtl *>(blk + sizeof(SweepDomain) * n);
    a.active = reinterpret_cast<int *>(a.ctl + 1);
    a.uoff = a.active + n;
    return QESB_OK;
  }
  // Uploads the domains (all active) and a fresh control block; returns once
  // the copies are done (the host-side sources may be locals).
  qesb_status upload(const std::vector<SweepDomain> &doms, int unit, cudaStream_t s)
  {
    const int n = (int)doms.size();
    if (n > cap) return qesb_fail(QESB_ERR_ARG, "domain list capacity %d < %d", cap, n);
    std::vector<int> active(n), uoff(n + 1, 0);
    for (int i = 0; i < n; ++i) {
      active[i] = i;
      uoff[i + 1] = uoff[i] + sweep_units(doms[i], unit);
    }
    const SweepCtl ctl{0u, n, 0, 0, 0ull};
    // the image in the staging buffer (the previous upload's copy has finished: it returned after it)
    const size_t o_ctl = (size_t)((unsigned char *)a.ctl - blk), o_act = (size_t)((unsigned char *)a.active - blk),
                 o_uoff = (size_t)((unsigned char *)a.uoff - blk);
    std::memcpy(stage, doms.data(), sizeof(SweepDomain) * n);
    std::memcpy(stage + o_ctl, &ctl, sizeof ctl);
    std::memcpy(stage + o_act, active.data(), sizeof(int) * n);
    std::memcpy(stage + o_uoff, uoff.data(), sizeof(int) * (n + 1));
    // everything but t0, the batch's start stamp (k_sweep_stamp), which outlives the pre-phase's list
    const size_t used = o_uoff + sizeof(int) * (n + 1);
    CKS(copy_words(blk, stage_dev, (used + 3) / 4 * 4, s, o_ctl + offsetof(SweepCtl, t0), o_ctl + sizeof(SweepCtl)));
    CK(cudaStreamSynchronize(s));
    return QESB_OK;
  }
  void destroy()
  {
    if (blk) cudaFree(blk);
    if (stage) cudaFreeHost(stage);
    blk = nullptr;
    stage = stage_dev = nullptr;
    cap = 0;
  }
};

// Graph cache of a handle: the captured chunk and what it was captured with.
struct SweepGraph {
  cudaGraphExec_t exec = nullptr;
  int variant = -1, chunk = 0;
  int wk = 0, nslots = 0;  // window checks captured: every wk launches, over nslots list slots
  bool multi = false;
  bool pdl = false;  // captured with programmatic dependent launches
  SweepArgs args{};
  cudaStream_t stream = nullptr;
  void reset()
  {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
  }
};

struct qesb_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  DevGrid G{};
  float dx = 1, dy = 1;
  std::vector<float> dz;
  float tol = 1e-9f;

  // device buffers
  float *d_lam = nullptr, *d_lam2 = nullptr;  // padded lambda (ping-pong for fused sweeps)
  float *d_R = nullptr;                       // padded R
  uint8_t *d_mask = nullptr;                  // padded wall mask
  float *d_pc[6] = {};                        // padded coefficients (full path)
  float *d_in[6] = {};                        // natural coefficients (owned copy, or caller's)
  int *d_flag = nullptr;
  float *d_u0 = nullptr, *d_v0 = nullptr, *d_w0 = nullptr;
  bool own_inputs = true;
  float *d_own_in[6] = {};
  int *d_own_flag = nullptr;
  float *d_own_u0 = nullptr, *d_own_v0 = nullptr, *d_own_w0 = nullptr;
  float *d_dz = nullptr;
  unsigned *d_vmax = nullptr;  // [6][Z] per-layer coefficient values (float bits)
  float *d_inv = nullptr;      // [Z][64] omega / sum
  float *d_val = nullptr;      // [6][Z] coefficient values
  int *d_bad = nullptr;
  double *d_err = nullptr;
  int err_cap = 0;
  SolveState *d_state = nullptr;
  SolveState *h_state = nullptr, *h_state_dev = nullptr;  // mapped pinned, and its device alias
  double *d_div = nullptr;        // final divergence check (FP64)
  float *d_u = nullptr, *d_v = nullptr, *d_w = nullptr;  // output staging for host solves
  cudaEvent_t ev[4] = {};
  cudaEvent_t evs[4] = {};  // around the sweep loops: pre-phase [0, 1], reference loop [2, 3]
  bool sweeps_timed = false;  // the last solve recorded evs

  bool have_inputs = false;
  bool packed = false;
  bool pc_ready = false;  // d_pc holds the current inputs' padded coefficients
  // R of the current inputs: inputs_gen counts input changes, R_gen the inputs d_R was computed from
  // (0: none, or inputs in caller-owned memory that may change behind the handle); ev_R follows it
  unsigned long long inputs_gen = 0, R_gen = 0;
  cudaEvent_t ev_R = nullptr;
  int opt_path = 1;
  int opt_k = 0;
  int opt_graph = 1;
  int opt_pdl = 0;  // programmatic dependent launches between z-march list kernels (measured: no gain)
  int opt_variant = -1;
  int opt_batch_variant = -1;  // sweep shape for batches led by this handle (qesb_autotune_batch)
  int opt_autotune = 0;
  unsigned opt_wait_limit = 0;  // staged sweeps' mbarrier polls before giving up (0: default)
  int last_launches = 0;

  // log-law wall treatment (qesb_wall_log_law): per-cell wall sides, cut-cell flag
  uint8_t *d_wbits = nullptr;
  int *d_wcut = nullptr;

  // red/black split layout (packed streaming path)
  SplitGeom S{};
  float *d_lam_s = nullptr, *d_R_s = nullptr;
  uint8_t *d_mask_s = nullptr;

  // over-relaxed pre-phase (qesb_set_prephase): omega 0 = off
  float pre_omega = 0.0f, pre_tol = 0.0f;
  int pre_iters = 0;
  float *d_inv_pre = nullptr;     // [Z][64] pre_omega / sum
  float inv_pre_omega = 0.0f;     // omega d_inv_pre holds (0 = stale)
  // start stage of the pre-phase: its first start_iters sweeps at start_omega
  float start_omega = 0.0f;
  int start_iters = 0;
  float *d_inv_start = nullptr;   // [Z][64] start_omega / sum
  float inv_start_omega = 0.0f;   // omega d_inv_start holds (0 = stale)
  int last_pre_iterations = 0;
  SweepGraph sgraph_pre;
  SweepGraph sgraph_start;

  // window rule (qesb_set_window_rule): window 0 = off
  int win_k = 0;
  double win_tol = 0.0;
  float *d_snap = nullptr;  // lambda at the start of the current window (split or padded layout)

  // tensor maps of the split arrays for the TMA z-march shapes: slot i holds
  // the kTmCount maps for tiles of tm_rows[i] rows (0: free). A slot is
  // encoded once and never rewritten, so captured graphs and lists in
  // flight keep valid maps whatever shape runs next.
  TmaDesc *d_tmaps = nullptr;
  int tm_rows[kTmSlots] = {};

  // sweep kernels: this solve as a one-domain list
  SweepList list;
  // batches led by this handle: their domain list and loop graphs, kept from
  // batch to batch (no allocation, free or graph instantiation per batch once warm)
  SweepList blist;
  SweepGraph bgraph_start, bgraph_pre, bgraph;
  SweepCtl *h_ctl = nullptr, *h_ctl_dev = nullptr;  // mapped pinned, and its device alias
  unsigned char *h_io = nullptr, *h_io_dev = nullptr;  // mapped pinned scratch for small reads (kIoBytes)
  SweepGraph sgraph;  // iteration-loop graph of the sweep kernels

  // iteration-loop graphs of the tiled path, one per (variant, starting buffer)
  struct GraphKey {
    int variant, start, chunk;
    float tol;
    int itermax;
    cudaStream_t stream;
  };
  GraphKey gkey[2] = {{-1, 0, 0, 0, 0, nullptr}, {-1, 1, 0, 0, 0, nullptr}};
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
};

namespace {

size_t pad_cells(const DevGrid &G) { return (size_t)G.PLANE * G.Z; }

// Tiled kernels read whole halo tiles; at the far x/y edge of the last
// plane a tile may run past the padded plane. The slack keeps those reads
// inside the allocation (the values read there feed only guard cells).
size_t pad_alloc(const DevGrid &G) { return pad_cells(G) + (size_t)(kMaxTileRows + kGY) * G.PX + 256; }

// ---------------------------------------------------------------------------
// tiled-kernel variants (template instances) and their launch shapes
// ---------------------------------------------------------------------------
struct Variant {
  const char *name;
  int K, BX, BY, NT, TX, TY;
  size_t smem;
  void (*fn)(TiledArgs);
};

template <int K, int BX, int BY, int NT>
constexpr Variant make_variant(const char *name)
{
  using C = TileCfg<K, BX, BY, NT>;
  return Variant{name, K, BX, BY, NT, C::TX, C::TY, C::SMEM, k_sor_tiled<K, BX, BY, NT>};
}

const Variant kVariants[] = {
    make_variant<1, 64, 32, 256>("k1_64x32"),
    make_variant<2, 64, 32, 256>("k2_64x32"),
    make_variant<2, 64, 48, 256>("k2_64x48"),
    make_variant<1, 128, 32, 512>("k1_128x32"),
    make_variant<2, 128, 24, 512>("k2_128x24"),
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);
static_assert(kMaxTileRows >= 48, "slack rows must cover the tallest tile");

qesb_status fill_grid(const qesb_grid *g, DevGrid &G)
{
  if (!g || g->Nx < 3 || g->Ny < 3 || g->Nz < 2 || !(g->dx > 0) || !(g->dy > 0) || !g->dz_array)
    return qesb_fail(QESB_ERR_ARG, "qesb_create: grid needs Nx, Ny >= 3, Nz >= 2, dx, dy > 0 and dz_array");
  if ((long)g->Nx * g->Ny * (g->Nz + 1) > (1L << 31) - 1)
    return qesb_fail(QESB_ERR_ARG, "qesb_create: grid too large for 32-bit cell indices");
  G.X = g->Nx;
  G.Y = g->Ny;
  G.Z = g->Nz + 1;
  G.FX = g->Nx + 1;
  G.FY = g->Ny + 1;
  G.FZ = g->Nz + 2;
  G.FXY = (long)G.FX * G.FY;
  G.XY = (long)G.X * G.Y;
  G.PX = ((G.X + 2 * kGX) + 31) / 32 * 32;
  G.PY = G.Y + 2 * kGY;
  G.PLANE = (long)G.PX * G.PY;
  for (int k = 0; k < G.Z; ++k)
    if (!(g->dz_array[k] > 0)) return qesb_fail(QESB_ERR_ARG, "qesb_create: dz_array[%d] must be > 0", k);
  return QESB_OK;
}

template <class T>
qesb_status dalloc(T **p, size_t count)
{
  CK(cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(count, 1)));
  return QESB_OK;
}

dim3 row_grid(const DevGrid &G, int rows, int planes, int width)
{
  return dim3((width + 255) / 256, rows, planes);
}

qesb_status ensure_err(qesb_handle *h, int itermax)
{
  if (h->err_cap >= itermax) return QESB_OK;
  if (h->d_err) cudaFree(h->d_err);
  h->d_err = nullptr;
  int cap = std::max(itermax, 1024);
  CKS(dalloc(&h->d_err, (size_t)cap));
  h->err_cap = cap;
  return QESB_OK;
}

// R of the handle's inputs into d_R: from the packed wall mask when the
// coefficients are stair-step, else from the six arrays (the same bits).
void launch_divergence(qesb_handle *h, cudaStream_t s)
{
  const DevGrid &G = h->G;
  if (h->packed)
    k_divergence_packed<<<row_grid(G, G.Y, G.Z - 2, G.X), 256, 0, s>>>(
        G, h->d_mask, h->d_val, h->d_in[0], h->d_in[1], h->d_in[2], h->d_in[3], h->d_in[4], h->d_in[5], h->d_u0,
        h->d_v0, h->d_w0, h->d_dz, h->dx, h->dy, h->d_R);
  else
    k_divergence<<<row_grid(G, G.Y, G.Z - 2, G.X), 256, 0, s>>>(G, h->d_in[0], h->d_in[1], h->d_in[2], h->d_in[3],
                                                                 h->d_in[4], h->d_in[5], h->d_u0, h->d_v0, h->d_w0,
                                                                 h->d_dz, h->dx, h->dy, h->d_R);
  // remembered for the next solve unless the inputs live in caller-owned memory
  h->R_gen = h->d_u0 == h->d_own_u0 && h->d_in[0] == h->d_own_in[0] ? h->inputs_gen : 0;
  cudaEventRecord(h->ev_R, s);
}

// Padded copies of the six coefficients for the full-coefficient sweep.
qesb_status ensure_padded_coefs(qesb_handle *h)
{
  if (h->pc_ready) return QESB_OK;
  const DevGrid &G = h->G;
  k_pad_coefs<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, h->stream>>>(
      G, h->d_in[0], h->d_in[1], h->d_in[2], h->d_in[3], h->d_in[4], h->d_in[5], h->d_pc[0], h->d_pc[1], h->d_pc[2],
      h->d_pc[3], h->d_pc[4], h->d_pc[5]);
  CK(cudaGetLastError());
  h->pc_ready = true;
  return QESB_OK;
}

// R for a solve: the R already computed from the same inputs (a warm start
// computes it first), ordered after its computation, or a new one.
void ensure_divergence(qesb_handle *h, cudaStream_t s)
{
  if (h->R_gen != 0 && h->R_gen == h->inputs_gen) cudaStreamWaitEvent(s, h->ev_R, 0);
  else launch_divergence(h, s);
}

// Inspect coefficients; build mask + tables when stair-step, else padded copies.
qesb_status prepare_coefs(qesb_handle *h)
{
  ++h->inputs_gen;  // new inputs: any R computed before is stale
  const DevGrid &G = h->G;
  cudaStream_t s = h->stream;
  h->packed = false;
  if (h->opt_path != 0) {
    CK(zero_async(h->d_vmax, sizeof(unsigned) * 6 * G.Z, s));
    CK(zero_async(h->d_bad, sizeof(int), s));
    k_layer_max<<<dim3((G.Y - 2 + 7) / 8, G.Z - 2), 256, 0, s>>>(G, h->d_in[0], h->d_in[1], h->d_in[2], h->d_in[3],
                                                                h->d_in[4], h->d_in[5], h->d_vmax, h->d_bad);
    CK(cudaGetLastError());
    k_build_mask<<<dim3(G.Y - 2, G.Z - 2), 256, 0, s>>>(G, h->d_in[0], h->d_in[1], h->d_in[2], h->d_in[3],
                                                         h->d_in[4], h->d_in[5], h->d_vmax, h->d_mask, h->d_bad);
    CK(cudaGetLastError());
    int bad = 1;
    CK(cudaMemcpyAsync(&bad, h->d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (!bad) {
      k_inv_table<<<G.Z, 64, 0, s>>>(G, h->d_vmax, h->d_inv, h->d_val, kOmega);
      h->inv_pre_omega = 0.0f;  // the pre-phase tables follow the new inputs at the next solve
      h->inv_start_omega = 0.0f;
      k_pad_to_split_u8<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, s>>>(G, h->S, h->d_mask, h->d_mask_s);
      CK(cudaGetLastError());
      h->packed = true;
    }
  }
  // The full-coefficient path (the sweep for non-stair-step inputs, and the
  // one the packed path is tested against) gets its padded copies here when
  // it is the only path, else at its first use.
  h->pc_ready = false;
  if (!h->packed) CKS(ensure_padded_coefs(h));
  return QESB_OK;
}

qesb_status run_iterations_full(qesb_handle *h, int itermax)
{
  CKS(ensure_padded_coefs(h));
  const DevGrid &G = h->G;
  cudaStream_t s = h->stream;
  const int nthr = 128;
  dim3 grid(((G.X - 2) / 2 + 1 + nthr - 1) / nthr, G.Y - 2, G.Z - 2);
  dim3 mgrid((G.X + 255) / 256, G.Y, 1);
  const int chunk = 64;
  const long n4 = (long)pad_cells(G) / 4;
  if (h->win_k > 0)  // the first window starts from lambda as the loop begins
    CKS(copy_floats(h->d_snap, h->d_lam, (long)pad_cells(G), s));
  for (int base = 0; base < itermax; base += chunk) {
    const int n = std::min(chunk, itermax - base);
    for (int t = 0; t < n; ++t) {
      for (int colour = 0; colour < 2; ++colour)
        k_sor_full<<<grid, nthr, 0, s>>>(G, colour, h->d_lam, h->d_pc[0], h->d_pc[1], h->d_pc[2],
                                         h->d_pc[3], h->d_pc[4], h->d_pc[5], h->d_R, h->d_err,
                                         h->d_state);
      k_mirror<<<mgrid, 256, 0, s>>>(G, h->d_lam, h->d_state);
      k_poll<<<1, 1, 0, s>>>(h->d_state, h->d_err, (double)h->tol, itermax, 1, 0);
      if (h->win_k > 0 && (base + t + 1) % h->win_k == 0) {
        k_window_full<<<592, 256, 0, s>>>(reinterpret_cast<const float4 *>(h->d_lam),
                                          reinterpret_cast<float4 *>(h->d_snap), n4, h->d_state);
        k_window_poll_full<<<1, 1, 0, s>>>(h->d_state, h->win_tol);
      }
    }
    CK(cudaGetLastError());
    CKS(copy_words(h->h_state_dev, h->d_state, sizeof(SolveState), s));
    CK(cudaStreamSynchronize(s));
    if (h->h_state->done) break;
  }
  return QESB_OK;
}

// Picks the tiled-kernel variant: the caller's sweeps_per_launch if set,
// else the autotuned choice for this grid (see autotune()).
int pick_variant(qesb_handle *h);
int tuned_variant(const DevGrid &G);

TiledArgs tiled_args(qesb_handle *h, const float *in, float *out, int itermax, int redo)
{
  TiledArgs a;
  a.G = h->G;
  a.lam_in = in;
  a.lam_out = out;
  a.R = h->d_R;
  a.mask = h->d_mask;
  a.val = h->d_val;
  a.inv = h->d_inv;
  a.err = h->d_err;
  a.st = h->d_state;
  a.itermax = itermax;
  a.redo = redo;
  return a;
}

dim3 tiled_grid(const DevGrid &G, const Variant &v)
{
  return dim3((G.X + v.TX - 1) / v.TX, (G.Y + v.TY - 1) / v.TY, 1);
}

qesb_status set_smem_attr(const Variant &v)
{
  static bool done[kNumVariants] = {};
  const int idx = (int)(&v - kVariants);
  if (!done[idx]) {
    CK(cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem));
    done[idx] = true;
  }
  return QESB_OK;
}

// One chunk of the tiled iteration loop: `chunk` launches alternating the two
// lambda buffers, each followed by its poll. Launches after the stop return
// at once (they read st->done first).
qesb_status enqueue_chunk(qesb_handle *h, const Variant &v, int start, int chunk, int itermax)
{
  cudaStream_t s = h->stream;
  float *buf[2] = {h->d_lam, h->d_lam2};
  const dim3 grid = tiled_grid(h->G, v);
  for (int c = 0; c < chunk; ++c) {
    const int src = (start + c) & 1, dst = src ^ 1;
    v.fn<<<grid, v.NT, v.smem, s>>>(tiled_args(h, buf[src], buf[dst], itermax, 0));
    k_poll<<<1, 1, 0, s>>>(h->d_state, h->d_err, (double)h->tol, itermax, v.K, dst);
  }
  CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status run_iterations_tiled(qesb_handle *h, const Variant &v, int itermax)
{
  cudaStream_t s = h->stream;
  CKS(set_smem_attr(v));
  // about 2 ms of device work per chunk between host polls of the state
  const double cells = (double)h->G.XY * h->G.Z;
  const int per_launch_us = std::max(1, (int)(cells * v.K / 4.0e5));
  int chunk = std::max(2, std::min(64, 2000 / per_launch_us));
  chunk += chunk & 1;  // even: every full chunk ends back in buffer 0
  const int max_launches = (itermax + v.K - 1) / v.K;
  int launched = 0;
  for (int base = 0; launched < max_launches; base += chunk) {
    if (h->opt_graph) {
      auto &key = h->gkey[0];
      const bool hit = h->gexec[0] && key.variant == (int)(&v - kVariants) && key.chunk == chunk &&
                       key.tol == h->tol && key.itermax == itermax && key.stream == s;
      if (!hit) {
        if (h->gexec[0]) cudaGraphExecDestroy(h->gexec[0]);
        h->gexec[0] = nullptr;
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        qesb_status qs = enqueue_chunk(h, v, 0, chunk, itermax);
        cudaError_t ce = cudaStreamEndCapture(s, &g);
        if (qs != QESB_OK) return qs;
        if (ce != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&h->gexec[0], g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
        key = {(int)(&v - kVariants), 0, chunk, h->tol, itermax, s};
      }
      CK(cudaGraphLaunch(h->gexec[0], s));
    } else {
      CKS(enqueue_chunk(h, v, 0, chunk, itermax));
    }
    launched += chunk;
    CKS(copy_words(h->h_state_dev, h->d_state, sizeof(SolveState), s));
    CK(cudaStreamSynchronize(s));
    if (h->h_state->done) break;
  }
  h->last_launches = launched * 2;
  // Exact stop: the converging launch fused iterations past the stop; re-run
  // only the iterations that count, from that launch's input buffer.
  if (h->h_state->redo > 0) {
    float *buf[2] = {h->d_lam, h->d_lam2};
    const int dst = h->h_state->redo_par;
    v.fn<<<tiled_grid(h->G, v), v.NT, v.smem, s>>>(tiled_args(h, buf[dst ^ 1], buf[dst], itermax, 1));
    CK(cudaGetLastError());
    h->last_launches += 1;
  }
  if (h->h_state->cur == 1) std::swap(h->d_lam, h->d_lam2);
  return QESB_OK;
}

// Red/black sweep launch shapes over domain lists: the streaming split
// kernels (rows per CTA, cells per lane, row order), the staged kernels
// (warps per CTA, stages per warp, copy engine) and the z-march kernels
// (rows per tile). unit: what the domain list counts (SweepUnit).
struct SweepVariant {
  const char *name;
  int unit;
  int block_y;  // warps per CTA
  int tile_rows;  // z-march tiles: rows per tile (0 for the other kinds)
  size_t smem;  // dynamic shared memory per CTA
  void (*red)(SweepArgs);  // single domain (from the kernel parameters)
  void (*black)(SweepArgs);
  void (*red_m)(SweepArgs);  // domain lists
  void (*black_m)(SweepArgs);
  int tma = 0;  // z-march shapes staged by tensor-map copies: the domains need their tensor maps
  int bal = 0;  // z-march shapes with equal plane-step shares per CTA (units of one plane: kc = 1)
};
// MINB: resident CTAs per SM the compiler must allow (caps registers per
// thread); the default allows 512 threads per SM (at most 128 registers)
template <int RPB, int U, int STRIDED = 0, int MINB = (16 / RPB > 1 ? 16 / RPB : 1)>
constexpr SweepVariant make_split(const char *name)
{
  return SweepVariant{name,
                      kUnitRow,
                      RPB,
                      0,
                      0,
                      k_sor_split<0, RPB, U, STRIDED, false, MINB>,
                      k_sor_split<1, RPB, U, STRIDED, false, MINB>,
                      k_sor_split<0, RPB, U, STRIDED, true, MINB>,
                      k_sor_split<1, RPB, U, STRIDED, true, MINB>};
}
template <int RPB, int STRIDED = 0, int MINB = (16 / RPB > 1 ? 16 / RPB : 1)>
constexpr SweepVariant make_split4(const char *name)
{
  return SweepVariant{name,
                      kUnitRow,
                      RPB,
                      0,
                      0,
                      k_sor_split4<0, RPB, STRIDED, false, MINB>,
                      k_sor_split4<1, RPB, STRIDED, false, MINB>,
                      k_sor_split4<0, RPB, STRIDED, true, MINB>,
                      k_sor_split4<1, RPB, STRIDED, true, MINB>};
}
template <int W, int NS, int ASYNC>
constexpr SweepVariant make_bulk(const char *name)
{
  return SweepVariant{name,
                      kUnitSpan,
                      W,
                      0,
                      bulk_smem_bytes<W, NS>(),
                      k_sor_bulk<0, W, NS, ASYNC, false>,
                      k_sor_bulk<1, W, NS, ASYNC, false>,
                      k_sor_bulk<0, W, NS, ASYNC, true>,
                      k_sor_bulk<1, W, NS, ASYNC, true>};
}
template <int TY, int RW, int MINB, int DIST = 2, int TMA = 0, int BAL = 0>
constexpr SweepVariant make_zm(const char *name)
{
  return SweepVariant{name,
                      kUnitTile,
                      TY,
                      TY * RW,
                      zm_smem_bytes<TY * RW, DIST, TMA>(),
                      k_sor_zm<0, TY, RW, DIST, false, MINB, TMA, BAL>,
                      k_sor_zm<1, TY, RW, DIST, false, MINB, TMA, BAL>,
                      k_sor_zm<0, TY, RW, DIST, true, MINB, TMA, BAL>,
                      k_sor_zm<1, TY, RW, DIST, true, MINB, TMA, BAL>,
                      TMA,
                      BAL};
}
const SweepVariant kSweepVariants[] = {
    // streaming split kernels (option "variant" 5..17)
    make_split<8, 4>("split_r8_u4"), make_split<8, 1>("split_r8_u1"), make_split<8, 2>("split_r8_u2"),
    make_split<4, 8>("split_r4_u8"), make_split<16, 2>("split_r16_u2"), make_split<4, 4, 0, 5>("split_r4_u4"),
    make_split4<4>("split4_r4"), make_split4<8>("split4_r8"), make_split4<16>("split4_r16"),
    make_split<4, 4, 1, 5>("split_r4_u4_strided"), make_split<8, 2, 1>("split_r8_u2_strided"),
    make_split4<4, 1>("split4_r4_strided"), make_split4<8, 1>("split4_r8_strided"),
    // staged kernels: bulk copies (18..22), per-lane async copies (23..27)
    make_bulk<4, 3, 0>("bulk_w4_s3"), make_bulk<4, 4, 0>("bulk_w4_s4"), make_bulk<4, 6, 0>("bulk_w4_s6"),
    make_bulk<8, 2, 0>("bulk_w8_s2"), make_bulk<8, 3, 0>("bulk_w8_s3"), make_bulk<4, 4, 1>("async_w4_s4"),
    make_bulk<8, 3, 1>("async_w8_s3"), make_bulk<4, 6, 1>("async_w4_s6"), make_bulk<16, 2, 1>("async_w16_s2"),
    make_bulk<8, 4, 1>("async_w8_s4"),
    // register-capped window-order shapes (28..31): more warps per SM for the same loads
    make_split4<8, 1, 3>("split4_r8_strided_b3"), make_split4<4, 1, 6>("split4_r4_strided_b6"),
    make_split<4, 4, 1, 6>("split_r4_u4_strided_b6"), make_split<8, 2, 1, 4>("split_r8_u2_strided_b4"),
    make_split4<8, 1, 4>("split4_r8_strided_b4"), make_split4<4, 1, 8>("split4_r4_strided_b8"),
    make_split4<16, 1, 2>("split4_r16_strided_b2"), make_split4<8, 0, 3>("split4_r8_b3"),
    // window order with an L2 prefetch of each warp's next row (36..39)
    make_split4<8, 2, 3>("split4_r8_pf_b3"), make_split4<4, 2, 6>("split4_r4_pf_b6"),
    make_split<4, 4, 2, 6>("split_r4_u4_pf_b6"), make_split4<4, 2, 8>("split4_r4_pf_b8"),
    // z-march tiles, other colour staged in shared memory (40..43)
    make_zm<8, 1, 4>("zm_y8"), make_zm<4, 1, 6>("zm_y4_b6"), make_zm<8, 1, 3>("zm_y8_b3"), make_zm<8, 1, 2>("zm_y8_b2"),
    // two rows per warp (44..47)
    make_zm<4, 2, 4>("zm_y4x2_b4"), make_zm<4, 2, 5>("zm_y4x2_b5"), make_zm<2, 2, 8>("zm_y2x2_b8"),
    make_zm<8, 2, 2>("zm_y8x2_b2"),
    // copies one plane ahead: smaller rings, more CTAs per SM (48..50)
    make_zm<4, 2, 5, 1>("zm_y4x2_d1_b5"), make_zm<4, 2, 4, 1>("zm_y4x2_d1_b4"), make_zm<2, 2, 8, 1>("zm_y2x2_d1_b8"),
    // the same staged by tensor-map copies issued from one thread (51..57; d2: two planes ahead)
    make_zm<4, 2, 5, 1, 1>("zmt_y4x2_b5"), make_zm<4, 2, 4, 1, 1>("zmt_y4x2_b4"), make_zm<2, 2, 8, 1, 1>("zmt_y2x2_b8"),
    make_zm<8, 2, 2, 1, 1>("zmt_y8x2_b2"), make_zm<4, 4, 2, 1, 1>("zmt_y4x4_b2"),
    make_zm<4, 2, 3, 2, 1>("zmt_y4x2_d2_b3"), make_zm<4, 2, 4, 2, 1>("zmt_y4x2_d2_b4"),
    // the same with equal plane-step shares per CTA (58..60)
    make_zm<4, 2, 4, 2, 1, 1>("zmtb_y4x2_d2_b4"), make_zm<4, 2, 5, 1, 1, 1>("zmtb_y4x2_b5"),
    make_zm<4, 2, 4, 1, 1, 1>("zmtb_y4x2_b4"),
};
constexpr int kNumSweep = sizeof(kSweepVariants) / sizeof(kSweepVariants[0]);
constexpr int kSplitVariant = kNumVariants;  // option "variant" index of the first sweep shape
constexpr int kAllVariants = kSplitVariant + kNumSweep;
constexpr int kDefaultSweep = 0;  // split_r8_u4 when nothing is tuned

qesb_status sweep_prepare(const SweepVariant &sv)
{
  if (sv.smem > 48 * 1024)
    for (auto fn : {sv.red, sv.black, sv.red_m, sv.black_m})
      CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sv.smem));
  return QESB_OK;
}

// Persistent grid: CTAs of the black kernel (the larger of the pair)
// resident at once on this device (occupancy x SMs), for the single-domain
// or the list instances.
int sweep_ctas(const SweepVariant &sv, bool multi, int device)
{
  static int nsm[64] = {};
  if (!nsm[device & 63]) cudaDeviceGetAttribute(&nsm[device & 63], cudaDevAttrMultiProcessorCount, device);
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, multi ? sv.black_m : sv.black, 32 * sv.block_y, sv.smem);
  return std::max(1, per) * std::max(1, nsm[device & 63]);
}

// Planes per z-march tile for a list: the kc in [4, 32] that minimises
// waves x (kc + 2) (the persistent grid's passes over the tiles, each costing
// its kc planes plus two staged halo planes), the same kc for every domain.
void sweep_tiles(std::vector<SweepDomain> &doms, const SweepVariant &sv, bool multi, int device)
{
  if (sv.unit != kUnitTile) return;
  if (sv.bal) {  // units of one plane of a tile column; the kernel splits them evenly over its CTAs
    for (SweepDomain &d : doms) {
      d.tile_y = sv.tile_rows;
      d.kc = 1;
    }
    return;
  }
  const long ctas = sweep_ctas(sv, multi, device);
  int best = 4;
  long best_cost = -1;
  for (int kc = 4; kc <= 32; ++kc) {
    long tiles = 0;
    for (SweepDomain &d : doms) {
      d.tile_y = sv.tile_rows;
      d.kc = kc;
      tiles += sweep_units(d, kUnitTile);
    }
    const long cost = (tiles + ctas - 1) / ctas * (kc + 2);
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best = kc;
    }
  }
  for (SweepDomain &d : doms) d.kc = best;
}

// cuTensorMapEncodeTiled, from the driver through the runtime (no libcuda link).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

qesb_status encode_tiled_fn(EncodeTiledFn *out)
{
  static EncodeTiledFn fn = nullptr;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess || !p ||
        q != cudaDriverEntryPointSuccess)
      return qesb_fail(QESB_ERR_CUDA, "cuTensorMapEncodeTiled not available");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  *out = fn;
  return QESB_OK;
}

// The handle's split arrays as 4-D tensors (q, j, k, colour) with the boxes
// the TMA z-march shapes copy for tiles of `rows` rows: the other colour's
// slab 136 x (rows + 2), the own colour's lambda and R 128 x rows (floats),
// the mask 128 x rows (bytes). Out-of-range elements read as zeros.
qesb_status ensure_tmaps(qesb_handle *h, int rows, cudaStream_t s, const TmaDesc **out)
{
  int slot = 0;
  while (slot < kTmSlots && h->tm_rows[slot] != 0 && h->tm_rows[slot] != rows) ++slot;
  if (slot == kTmSlots) return qesb_fail(QESB_ERR_ARG, "more than %d tile heights with tensor maps", kTmSlots);
  if (h->tm_rows[slot] == rows) {
    *out = h->d_tmaps + slot * kTmCount;
    return QESB_OK;
  }
  EncodeTiledFn enc = nullptr;
  CKS(encode_tiled_fn(&enc));
  if (!h->d_tmaps) CKS(dalloc(&h->d_tmaps, kTmCount * kTmSlots));
  TmaDesc maps_h[kTmCount];
  const cuuint64_t dims[4] = {(cuuint64_t)h->S.PQ, (cuuint64_t)h->G.Y, (cuuint64_t)h->G.Z, 2};
  const cuuint64_t fstr[3] = {(cuuint64_t)h->S.PQ * 4, (cuuint64_t)h->S.PQ * h->G.Y * 4, (cuuint64_t)h->S.CS * 4};
  const cuuint64_t bstr[3] = {(cuuint64_t)h->S.PQ, (cuuint64_t)h->S.PQ * h->G.Y, (cuuint64_t)h->S.CS};
  const cuuint32_t one[4] = {1, 1, 1, 1};
  const cuuint32_t box_oth[4] = {(cuuint32_t)kZmOW, (cuuint32_t)rows + 2, 1, 1};
  const cuuint32_t box_own[4] = {(cuuint32_t)kZmQ, (cuuint32_t)rows, 1, 1};
  struct M {
    CUtensorMapDataType t;
    void *base;
    const cuuint64_t *str;
    const cuuint32_t *box;
  } maps[kTmCount] = {{CU_TENSOR_MAP_DATA_TYPE_FLOAT32, h->d_lam_s, fstr, box_oth},
                      {CU_TENSOR_MAP_DATA_TYPE_FLOAT32, h->d_lam_s, fstr, box_own},
                      {CU_TENSOR_MAP_DATA_TYPE_FLOAT32, h->d_R_s, fstr, box_own},
                      {CU_TENSOR_MAP_DATA_TYPE_UINT8, h->d_mask_s, bstr, box_own}};
  static_assert(sizeof(CUtensorMap) == sizeof(TmaDesc), "tensor map size");
  for (int q = 0; q < kTmCount; ++q) {
    CUtensorMap m;
    const CUresult r = enc(&m, maps[q].t, 4, maps[q].base, dims, maps[q].str, maps[q].box, one,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return qesb_fail(QESB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) for map %d", (int)r, q);
    std::memcpy(&maps_h[q], &m, sizeof m);
  }
  // on the stream of the launches that read them; from pageable memory, so
  // maps_h may go out of scope when the call returns
  CK(cudaMemcpyAsync(h->d_tmaps + slot * kTmCount, maps_h, sizeof maps_h, cudaMemcpyHostToDevice, s));
  h->tm_rows[slot] = rows;
  *out = h->d_tmaps + slot * kTmCount;
  return QESB_OK;
}

// The domain's tensor maps for a TMA shape (no-op for the others); s is the
// stream of the launches that use them.
qesb_status attach_tmaps(qesb_handle *h, const SweepVariant &sv, SweepDomain &d, cudaStream_t s)
{
  if (!sv.tma) return QESB_OK;
  const TmaDesc *m = nullptr;
  CKS(ensure_tmaps(h, sv.tile_rows, s, &m));
  d.tm = m;
  return QESB_OK;
}

SweepDomain sweep_domain(qesb_handle *h, int itermax, double tol)
{
  const DevGrid &G = h->G;
  SweepDomain d{};
  d.X = G.X;
  d.Y = G.Y;
  d.Z = G.Z;
  d.PQ = h->S.PQ;
  d.CS = h->S.CS;
  d.nch = (h->S.PQ + kChunk - 1) / kChunk;
  d.rows = (G.Y - 2) * (G.Z - 2);
  d.lam = h->d_lam_s;
  d.R = h->d_R_s;
  d.mask = h->d_mask_s;
  d.val = h->d_val;
  d.inv = h->d_inv;
  d.err = h->d_err;
  d.st = h->d_state;
  d.itermax = itermax;
  d.tol = tol;
  d.c1 = 1.0f - kOmega;
  d.wK = h->win_k;
  d.wn = 2 * h->S.CS;
  d.wtol = h->win_tol;
  d.snap = h->d_snap;
  return d;
}

// The pre-phase's view of a domain: omega = pre_omega through its own inv
// table and c1, its own tolerance and iteration cap.
qesb_status sweep_domain_pre(qesb_handle *h, SweepDomain &d, cudaStream_t s)
{
  if (h->inv_pre_omega != h->pre_omega) {
    k_inv_table<<<h->G.Z, 64, 0, s>>>(h->G, h->d_vmax, h->d_inv_pre, h->d_val, h->pre_omega);
    CK(cudaGetLastError());
    h->inv_pre_omega = h->pre_omega;
  }
  d = sweep_domain(h, h->pre_iters, (double)h->pre_tol);
  d.inv = h->d_inv_pre;
  d.c1 = 1.0f - h->pre_omega;
  d.wK = 0;  // the window rule ends the reference loop only
  return QESB_OK;
}

// The pre-phase's start stage: start_iters sweeps at start_omega, no stop
// on the tolerance (its own inv table, 1 - start_omega).
qesb_status sweep_domain_start(qesb_handle *h, SweepDomain &d, cudaStream_t s)
{
  if (h->inv_start_omega != h->start_omega) {
    k_inv_table<<<h->G.Z, 64, 0, s>>>(h->G, h->d_vmax, h->d_inv_start, h->d_val, h->start_omega);
    CK(cudaGetLastError());
    h->inv_start_omega = h->start_omega;
  }
  d = sweep_domain(h, h->start_iters, -1.0);  // tol < 0: every sweep runs
  d.inv = h->d_inv_start;
  d.c1 = 1.0f - h->start_omega;
  d.wK = 0;
  return QESB_OK;
}

// Whether the handle's next solve runs a pre-phase, and a start stage in it.
bool prephase_on(const qesb_handle *h) { return h->pre_omega > 0.0f && h->pre_iters > 0; }
bool start_on(const qesb_handle *h) { return prephase_on(h) && h->start_omega > 0.0f && h->start_iters > 0; }
int err_slots(const qesb_handle *h, int itermax)
{
  return std::max({itermax, 1, prephase_on(h) ? h->pre_iters : 0, start_on(h) ? h->start_iters : 0});
}

// Window check launch for a list of kernels of work-unit kind `unit`.
// A list kernel launch, as a programmatic dependent launch when pdl is set
// (the kernel starts with pdl_wait_release()).
cudaError_t launch_list(void (*k)(SweepArgs), dim3 grid, dim3 block, size_t smem, cudaStream_t s, const SweepArgs &a,
                        bool pdl)
{
  if (!pdl) {
    k<<<grid, block, smem, s>>>(a);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, a);
}

void launch_window(int unit, bool multi, dim3 grid, cudaStream_t s, const SweepArgs &a, bool pdl = false)
{
  void (*k)(SweepArgs) = unit == kUnitTile   ? (multi ? k_window_check<kUnitTile, true> : k_window_check<kUnitTile, false>)
                         : unit == kUnitSpan ? (multi ? k_window_check<kUnitSpan, true> : k_window_check<kUnitSpan, false>)
                                             : (multi ? k_window_check<kUnitRow, true> : k_window_check<kUnitRow, false>);
  launch_list(k, grid, dim3(256), 0, s, a, pdl);
}

// The iteration loop over a domain list: CUDA-graph chunks of (red, black)
// launches, the list's control block read back every ~2 ms of device work,
// until no domain is left or itermax launches ran. *launched: iterations
// launched. wk > 0: a window check (k_window_check over `nslots` list slots)
// follows every wk-th black launch; chunks are then whole windows, so the
// checks fall on iterations wk, 2 wk, ... of the loop for every domain.
qesb_status run_sweep_loop(const SweepVariant &sv, bool multi, const SweepArgs &a, int device, cudaStream_t s,
                           double cells, int itermax, bool graph, SweepGraph *cache, SweepCtl *h_ctl,
                           SweepCtl *h_ctl_dev, int *launched,
                           int wk = 0, int nslots = 1, bool pdl = false)
{
  CKS(sweep_prepare(sv));
  const dim3 grid(sweep_ctas(sv, multi, device)), block(32, sv.block_y);
  const int per_it_us = std::max(1, (int)(cells / 4.0e5));
  int chunk = std::max(1, std::min(128, 2000 / per_it_us));
  if (wk > 0) chunk = wk * std::max(1, chunk / wk);
  else chunk = std::max(1, std::min(chunk, itermax));  // a short fixed phase (a start stage) launches no empty tail
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const dim3 wgrid(std::max(1, 4 * sms / std::max(1, nslots)), std::max(1, nslots));
  auto red = multi ? sv.red_m : sv.red, black = multi ? sv.black_m : sv.black;
  // programmatic dependent launches between the z-march list kernels (the
  // first of a chunk waits for the chunk before it in the usual way)
  const bool chain = pdl && sv.tile_rows > 0;
  auto enqueue = [&]() {
    cudaError_t e = cudaSuccess;
    for (int c = 0; c < chunk && e == cudaSuccess; ++c) {
      e = launch_list(red, grid, block, sv.smem, s, a, chain && c > 0);
      if (e == cudaSuccess) e = launch_list(black, grid, block, sv.smem, s, a, chain);
      if (e == cudaSuccess && wk > 0 && (c + 1) % wk == 0) launch_window(sv.unit, multi, wgrid, s, a, chain);
    }
    return e != cudaSuccess ? e : cudaGetLastError();
  };
  const int vid = (int)(&sv - kSweepVariants);
  *launched = 0;
  while (*launched < itermax) {
    if (graph) {
      const bool hit = cache->exec && cache->variant == vid && cache->chunk == chunk && cache->multi == multi &&
                       cache->wk == wk && cache->nslots == nslots && cache->stream == s && cache->pdl == chain &&
                       std::memcmp(&cache->args, &a, sizeof a) == 0;
      if (!hit) {
        cache->reset();
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        cudaError_t qe = enqueue();
        cudaError_t ce = cudaStreamEndCapture(s, &g);
        if (qe != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "sweep launch: %s", cudaGetErrorString(qe));
        if (ce != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&cache->exec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
        cache->variant = vid;
        cache->chunk = chunk;
        cache->wk = wk;
        cache->nslots = nslots;
        cache->multi = multi;
        cache->pdl = chain;
        cache->stream = s;
        std::memcpy(&cache->args, &a, sizeof a);
      }
      CK(cudaGraphLaunch(cache->exec, s));
    } else {
      CK(enqueue());
    }
    *launched += chunk;
    CKS(copy_words(h_ctl_dev, a.ctl, sizeof(SweepCtl), s));
    CK(cudaStreamSynchronize(s));
    if (h_ctl->fault) return qesb_fail(QESB_ERR_CUDA, "sweep stage wait gave up");
    if (h_ctl->nactive == 0) break;
  }
  return QESB_OK;
}

// One solve on the sweep kernels: lambda and R to the split layout, the
// loop over a one-domain list, then the boundary-ring mirror and lambda back.
qesb_status run_iterations_sweep(qesb_handle *h, const SweepVariant &sv, int itermax)
{
  const DevGrid &G = h->G;
  cudaStream_t s = h->stream;
  k_pad_to_split<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, s>>>(G, h->S, h->d_lam, h->d_lam_s);
  k_pad_to_split<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, s>>>(G, h->S, h->d_R, h->d_R_s);
  CK(cudaGetLastError());
  int launched = 0, pre_launched = 0;
  h->last_pre_iterations = 0;
  CK(cudaEventRecord(h->evs[0], s));
  if (start_on(h)) {
    // the pre-phase's start stage: start_iters sweeps at start_omega
    std::vector<SweepDomain> st1(1);
    CKS(sweep_domain_start(h, st1[0], s));
    CKS(attach_tmaps(h, sv, st1[0], s));
    sweep_tiles(st1, sv, false, h->device);
    CKS(h->list.upload(st1, sv.unit, s));
    SweepArgs a = h->list.a;
    a.one = st1[0];
    a.wait_limit = h->opt_wait_limit;
    int n1 = 0;
    CKS(run_sweep_loop(sv, false, a, h->device, s, (double)G.XY * G.Z, h->start_iters, h->opt_graph != 0,
                       &h->sgraph_start, h->h_ctl, h->h_ctl_dev, &n1, 0, 1, h->opt_pdl != 0));
    pre_launched += n1;
    CKS(copy_words(h->h_state_dev, h->d_state, sizeof(SolveState), s));
    CK(cudaStreamSynchronize(s));
    if (h->h_state->nan) return qesb_fail(QESB_ERR_NUMERIC, "NaN in lambda during the pre-phase's start stage");
    h->last_pre_iterations = h->h_state->it;
    CK(zero_async(h->d_err, sizeof(double) * err_slots(h, itermax), s));
    CK(zero_async(h->d_state, sizeof(SolveState), s));
  }
  if (prephase_on(h)) {
    // over-relaxed pre-phase from the current lambda; its state and error
    // history are then cleared for the reference loop
    std::vector<SweepDomain> pre(1);
    CKS(sweep_domain_pre(h, pre[0], s));
    CKS(attach_tmaps(h, sv, pre[0], s));
    sweep_tiles(pre, sv, false, h->device);
    CKS(h->list.upload(pre, sv.unit, s));
    SweepArgs a = h->list.a;
    a.one = pre[0];
    a.wait_limit = h->opt_wait_limit;
    int n2 = 0;
    CKS(run_sweep_loop(sv, false, a, h->device, s, (double)G.XY * G.Z, h->pre_iters, h->opt_graph != 0,
                       &h->sgraph_pre, h->h_ctl, h->h_ctl_dev, &n2, 0, 1, h->opt_pdl != 0));
    pre_launched += n2;
    CKS(copy_words(h->h_state_dev, h->d_state, sizeof(SolveState), s));
    CK(cudaStreamSynchronize(s));
    if (h->h_state->nan) return qesb_fail(QESB_ERR_NUMERIC, "NaN in lambda during the pre-phase");
    h->last_pre_iterations += h->h_state->it;
    CK(zero_async(h->d_err, sizeof(double) * std::max(itermax, 1), s));
    CK(zero_async(h->d_state, sizeof(SolveState), s));
  }
  CK(cudaEventRecord(h->evs[1], s));
  std::vector<SweepDomain> one{sweep_domain(h, itermax, (double)h->tol)};
  CKS(attach_tmaps(h, sv, one[0], s));
  sweep_tiles(one, sv, false, h->device);
  CKS(h->list.upload(one, sv.unit, s));
  SweepArgs a = h->list.a;
  a.one = one[0];
  a.wait_limit = h->opt_wait_limit;
  if (h->win_k > 0)  // the first window starts from lambda as the reference loop begins
    CKS(copy_floats(h->d_snap, h->d_lam_s, 2L * h->S.CS, s));
  CK(cudaEventRecord(h->evs[2], s));
  CKS(run_sweep_loop(sv, false, a, h->device, s, (double)G.XY * G.Z, itermax, h->opt_graph != 0, &h->sgraph,
                     h->h_ctl, h->h_ctl_dev, &launched, h->win_k, 1, h->opt_pdl != 0));
  CK(cudaEventRecord(h->evs[3], s));
  h->sweeps_timed = true;
  h->last_launches = 2 * (launched + pre_launched) + (h->win_k > 0 ? launched / h->win_k : 0);
  k_split_mirror_ring<<<G.Y, 128, 0, s>>>(G, h->S, h->d_lam_s);
  k_split_to_pad<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, s>>>(G, h->S, h->d_lam_s, h->d_lam);
  CK(cudaGetLastError());
  h->last_launches += 5;
  return QESB_OK;
}

// FP64 final divergence check of (u, v, w) into h->d_div (all three needed).
qesb_status enqueue_divergence_check(qesb_handle *h, const float *u, const float *v, const float *w, cudaStream_t s)
{
  const DevGrid &G = h->G;
  CK(zero_async(h->d_div, sizeof(double), s));
  const int kmax = G.FZ - 4;
  if (kmax >= 1) {
    k_max_divergence<<<dim3(1, (G.Y - 2 + 7) / 8, kmax), dim3(32, 8), 0, s>>>(G, h->d_flag, u, v, w, h->d_dz, h->dx,
                                                                             h->dy, kmax, h->d_div);
    CK(cudaGetLastError());
  }
  return QESB_OK;
}

qesb_status solve_impl(qesb_handle *h, int itermax, float *u, float *v, float *w, qesb_stats *st)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  if (!h->have_inputs) return qesb_fail(QESB_ERR_STATE, "qesb_solve before qesb_set_inputs");
  if (itermax < 0) return qesb_fail(QESB_ERR_ARG, "itermax must be >= 0");
  CK(cudaSetDevice(h->device));
  const DevGrid &G = h->G;
  cudaStream_t s = h->stream;
  const int nerr = err_slots(h, itermax);
  CKS(ensure_err(h, nerr));
  CK(cudaEventRecord(h->ev[0], s));
  ensure_divergence(h, s);
  CK(cudaGetLastError());
  CK(zero_async(h->d_err, sizeof(double) * nerr, s));
  CK(zero_async(h->d_state, sizeof(SolveState), s));
  CK(cudaEventRecord(h->ev[1], s));
  const bool packed = h->packed && h->opt_path == 1;
  if (packed && h->opt_autotune && h->opt_variant < 0 && tuned_variant(G) < 0) {
    CKS(qesb_autotune(h, nullptr, nullptr, 0));
    CK(cudaEventRecord(h->ev[1], s));
  }
  int vi = packed ? pick_variant(h) : -1;
  // the fused tiled kernels have no window checks and no pre-phase: either runs on the sweep kernels
  if (packed && (h->win_k > 0 || prephase_on(h)) && vi < kSplitVariant) vi = kSplitVariant + kDefaultSweep;
  const bool split = packed && vi >= kSplitVariant;
  const Variant *var = packed && !split ? &kVariants[vi] : nullptr;
  h->last_launches = 0;
  h->last_pre_iterations = 0;
  h->sweeps_timed = false;
  if (itermax > 0) {
    if (split) CKS(run_iterations_sweep(h, kSweepVariants[vi - kSplitVariant], itermax));
    else if (var) CKS(run_iterations_tiled(h, *var, itermax));
    else CKS(run_iterations_full(h, itermax));
  }
  CK(cudaEventRecord(h->ev[2], s));
  k_correct<<<dim3(1, (G.FY + 7) / 8, G.FZ), dim3(32, 8), 0, s>>>(
      G, h->d_lam, h->d_in[1], h->d_in[3], h->d_in[5], h->d_flag, h->d_u0, h->d_v0, h->d_w0,
      h->d_dz, h->dx, h->dy, u, v, w);
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev[3], s));
  const bool check = u && v && w;
  if (check) CKS(enqueue_divergence_check(h, u, v, w, s));
  double div = -1.0;
  if (check) CKS(copy_words(h->h_io_dev, h->d_div, sizeof(double), s));
  CKS(copy_words(h->h_state_dev, h->d_state, sizeof(SolveState), s));
  CK(cudaStreamSynchronize(s));
  if (check) std::memcpy(&div, h->h_io, sizeof div);
  if (st) {
    st->max_divergence = div;
    float a = 0, b = 0;
    CK(cudaEventElapsedTime(&a, h->ev[0], h->ev[3]));
    CK(cudaEventElapsedTime(&b, h->ev[1], h->ev[2]));
    st->iterations = itermax > 0 ? h->h_state->it : 0;
    st->converged = h->h_state->converged;
    st->residual = itermax > 0 ? h->h_state->residual : 1.0;
    st->ms_total = a;
    st->ms_sor = b;
    st->path = packed ? 1 : 0;
    st->sweeps_per_launch = var ? var->K : 1;
    st->launches = 2 + (packed ? h->last_launches : 4 * st->iterations);
    st->pre_iterations = h->last_pre_iterations;
    st->window_drift = h->win_k > 0 && st->iterations >= h->win_k ? h->h_state->wdrift : -1.0;
    st->ms_sweeps = -1.0;
    if (h->sweeps_timed) {
      float p = 0, r = 0;
      CK(cudaEventElapsedTime(&p, h->evs[0], h->evs[1]));
      CK(cudaEventElapsedTime(&r, h->evs[2], h->evs[3]));
      st->ms_sweeps = (double)p + (double)r;
    }
  }
  if (h->h_state->nan) return qesb_fail(QESB_ERR_NUMERIC, "NaN in lambda during the solve (iteration %d)", h->h_state->it);
  return QESB_OK;
}

// Process-wide autotuner choices, per grid shape.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int> g_tuned;

int tuned_variant(const DevGrid &G)
{
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find({G.X, G.Y, G.Z});
  return it == g_tuned.end() ? -1 : it->second;
}

int pick_variant(qesb_handle *h)
{
  if (h->opt_variant >= 0) return h->opt_variant;
  if (h->opt_k == 2) return 1;  // fused: K = 2, 64 x 32 tiles
  const int t = tuned_variant(h->G);
  if (t >= 0) return t;
  return kSplitVariant;         // streaming red/black split half-sweeps
}

void free_all(qesb_handle *h)
{
  for (auto &g : h->gexec)
    if (g) cudaGraphExecDestroy(g);
  h->sgraph.reset();
  h->sgraph_pre.reset();
  h->sgraph_start.reset();
  void *ptrs[] = {h->d_lam_s, h->d_R_s, h->d_mask_s, h->d_lam, h->d_lam2, h->d_R, h->d_mask, h->d_pc[0], h->d_pc[1], h->d_pc[2],
                  h->d_pc[3], h->d_pc[4], h->d_pc[5], h->d_own_in[0], h->d_own_in[1],
                  h->d_own_in[2], h->d_own_in[3], h->d_own_in[4], h->d_own_in[5], h->d_own_flag,
                  h->d_own_u0, h->d_own_v0, h->d_own_w0, h->d_dz, h->d_vmax, h->d_inv, h->d_val,
                  h->d_inv_pre, h->d_inv_start, h->d_bad, h->d_err, h->d_state, h->d_u, h->d_v, h->d_w, h->d_wbits,
                  h->d_wcut, h->d_snap, h->d_tmaps};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  h->list.destroy();
  h->blist.destroy();
  h->bgraph_start.reset();
  h->bgraph_pre.reset();
  h->bgraph.reset();
  if (h->h_state) cudaFreeHost(h->h_state);
  if (h->h_ctl) cudaFreeHost(h->h_ctl);
  if (h->h_io) cudaFreeHost(h->h_io);
  for (auto &e : h->ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : h->evs)
    if (e) cudaEventDestroy(e);
  if (h->ev_R) cudaEventDestroy(h->ev_R);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char *qesb_version(void) { return "qesb200 0.1 (sm_100a)"; }
const char *qesb_last_error(void) { return g_last_error.c_str(); }

qesb_status qesb_create(const qesb_grid *grid, float tol, int device, qesb_handle **out)
{
  if (!out) return qesb_fail(QESB_ERR_ARG, "qesb_create: null out");
  *out = nullptr;
  DevGrid G{};
  CKS(fill_grid(grid, G));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return qesb_fail(QESB_ERR_NODEV, "qesb_create: no CUDA device");
  if (device < 0 || device >= ndev) return qesb_fail(QESB_ERR_ARG, "qesb_create: device %d out of range", device);
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) return qesb_fail(QESB_ERR_NODEV, "qesb_create: device %d is sm_%d%d, this build is sm_100a", device, prop.major, prop.minor);
  CK(cudaSetDevice(device));
  qesb_handle *h = new qesb_handle();
  h->device = device;
  h->G = G;
  h->dx = grid->dx;
  h->dy = grid->dy;
  h->dz.assign(grid->dz_array, grid->dz_array + G.Z);
  h->tol = tol;
  auto fail = [&](qesb_status s) {
    free_all(h);
    delete h;
    return s;
  };
  qesb_status s = QESB_OK;
#define TRY(x)                          \
  if ((s = (x)) != QESB_OK) return fail(s);
  const size_t np = pad_alloc(G), nc = (size_t)G.XY * G.Z, nf = (size_t)G.FXY * G.FZ;
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(qesb_fail(QESB_ERR_CUDA, "cudaStreamCreate failed"));
  h->stream = h->own_stream;
  TRY(dalloc(&h->d_lam, np));
  TRY(dalloc(&h->d_lam2, np));
  TRY(dalloc(&h->d_R, np));
  TRY(dalloc(&h->d_mask, np));
  for (int q = 0; q < 6; ++q) TRY(dalloc(&h->d_pc[q], np));
  h->S.PQ = ((G.X + 1) / 2 + 31) / 32 * 32;
  h->S.CS = (long)h->S.PQ * G.Y * G.Z;
  TRY(dalloc(&h->d_lam_s, 2 * h->S.CS));
  TRY(dalloc(&h->d_R_s, 2 * h->S.CS));
  TRY(dalloc(&h->d_mask_s, 2 * h->S.CS));
  TRY(dalloc(&h->d_dz, G.Z));
  TRY(dalloc(&h->d_vmax, 6 * G.Z));
  TRY(dalloc(&h->d_inv, 64 * G.Z));
  TRY(dalloc(&h->d_inv_pre, 64 * G.Z));
  TRY(dalloc(&h->d_inv_start, 64 * G.Z));
  TRY(dalloc(&h->d_val, 6 * G.Z));
  TRY(dalloc(&h->d_bad, 1));
  TRY(dalloc(&h->d_state, 1));
  TRY(dalloc(&h->d_div, 1));
  TRY(h->list.create(1));
  TRY(ensure_err(h, 1024));
  TRY(host_mapped(&h->h_state, &h->h_state_dev, sizeof(SolveState)));
  TRY(host_mapped(&h->h_ctl, &h->h_ctl_dev, sizeof(SweepCtl)));
  TRY(host_mapped(&h->h_io, &h->h_io_dev, kIoBytes));
  for (auto &e : h->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(qesb_fail(QESB_ERR_CUDA, "cudaEventCreate failed"));
  for (auto &e : h->evs)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(qesb_fail(QESB_ERR_CUDA, "cudaEventCreate failed"));
  if (cudaEventCreateWithFlags(&h->ev_R, cudaEventDisableTiming) != cudaSuccess)
    return fail(qesb_fail(QESB_ERR_CUDA, "cudaEventCreate failed"));
  for (void *p : {(void *)h->d_lam, (void *)h->d_lam2, (void *)h->d_R})
    if (cudaMemset(p, 0, np * sizeof(float)) != cudaSuccess) return fail(qesb_fail(QESB_ERR_CUDA, "cudaMemset failed"));
  if (cudaMemset(h->d_mask, 0, np) != cudaSuccess) return fail(qesb_fail(QESB_ERR_CUDA, "cudaMemset failed"));
  if (cudaMemset(h->d_lam_s, 0, 2 * h->S.CS * sizeof(float)) != cudaSuccess ||
      cudaMemset(h->d_R_s, 0, 2 * h->S.CS * sizeof(float)) != cudaSuccess ||
      cudaMemset(h->d_mask_s, 0, 2 * h->S.CS) != cudaSuccess)
    return fail(qesb_fail(QESB_ERR_CUDA, "cudaMemset failed"));
  for (int q = 0; q < 6; ++q)
    if (cudaMemset(h->d_pc[q], 0, np * sizeof(float)) != cudaSuccess) return fail(qesb_fail(QESB_ERR_CUDA, "cudaMemset failed"));
  if (cudaMemcpy(h->d_dz, h->dz.data(), sizeof(float) * G.Z, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(qesb_fail(QESB_ERR_CUDA, "cudaMemcpy dz failed"));
  (void)nc;
  (void)nf;
#undef TRY
  *out = h;
  return QESB_OK;
}

qesb_status qesb_destroy(qesb_handle *h)
{
  if (!h) return QESB_OK;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
  return QESB_OK;
}

qesb_status qesb_reset_lambda(qesb_handle *h)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  CK(cudaSetDevice(h->device));
  const size_t np = pad_alloc(h->G);
  CK(zero_async(h->d_lam, np * sizeof(float), h->stream));
  CK(zero_async(h->d_lam2, np * sizeof(float), h->stream));
  CK(zero_async(h->d_R, np * sizeof(float), h->stream));
  h->R_gen = 0;  // R is recomputed by the next solve
  CK(cudaStreamSynchronize(h->stream));
  return QESB_OK;
}

static qesb_status ensure_own_inputs(qesb_handle *h)
{
  const size_t nc = (size_t)h->G.XY * h->G.Z, nf = (size_t)h->G.FXY * h->G.FZ;
  for (int q = 0; q < 6; ++q)
    if (!h->d_own_in[q]) CKS(dalloc(&h->d_own_in[q], nc));
  if (!h->d_own_flag) CKS(dalloc(&h->d_own_flag, nc));
  if (!h->d_own_u0) CKS(dalloc(&h->d_own_u0, nf));
  if (!h->d_own_v0) CKS(dalloc(&h->d_own_v0, nf));
  if (!h->d_own_w0) CKS(dalloc(&h->d_own_w0, nf));
  return QESB_OK;
}

qesb_status qesb_set_inputs(qesb_handle *h, const float *e, const float *f, const float *g,
                            const float *hc, const float *m, const float *n, const int *icellflag,
                            const float *u0, const float *v0, const float *w0)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  if (!e || !f || !g || !hc || !m || !n || !icellflag || !u0 || !v0 || !w0)
    return qesb_fail(QESB_ERR_ARG, "qesb_set_inputs: null input");
  CK(cudaSetDevice(h->device));
  CKS(ensure_own_inputs(h));
  const size_t nc = (size_t)h->G.XY * h->G.Z, nf = (size_t)h->G.FXY * h->G.FZ;
  const float *src[6] = {e, f, g, hc, m, n};
  cudaStream_t s = h->stream;
  for (int q = 0; q < 6; ++q) CK(cudaMemcpyAsync(h->d_own_in[q], src[q], nc * sizeof(float), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_own_flag, icellflag, nc * sizeof(int), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_own_u0, u0, nf * sizeof(float), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_own_v0, v0, nf * sizeof(float), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_own_w0, w0, nf * sizeof(float), cudaMemcpyHostToDevice, s));
  for (int q = 0; q < 6; ++q) h->d_in[q] = h->d_own_in[q];
  h->d_flag = h->d_own_flag;
  h->d_u0 = h->d_own_u0;
  h->d_v0 = h->d_own_v0;
  h->d_w0 = h->d_own_w0;
  CKS(prepare_coefs(h));
  CK(cudaStreamSynchronize(s));
  h->have_inputs = true;
  return QESB_OK;
}

qesb_status qesb_set_inputs_flags(qesb_handle *h, const int *icellflag, const float *u0, const float *v0,
                                  const float *w0)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  if (!icellflag || !u0 || !v0 || !w0) return qesb_fail(QESB_ERR_ARG, "qesb_set_inputs_flags: null input");
  CK(cudaSetDevice(h->device));
  CKS(ensure_own_inputs(h));
  const size_t nc = (size_t)h->G.XY * h->G.Z, nf = (size_t)h->G.FXY * h->G.FZ;
  cudaStream_t s = h->stream;
  CK(cudaMemcpyAsync(h->d_own_flag, icellflag, nc * sizeof(int), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_own_u0, u0, nf * sizeof(float), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_own_v0, v0, nf * sizeof(float), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_own_w0, w0, nf * sizeof(float), cudaMemcpyHostToDevice, s));
  CKS(qesb_city_walls_dev(h->G.X, h->G.Y, h->G.Z - 1, h->dx, h->d_dz, h->d_own_flag, h->d_own_in[0], h->d_own_in[1],
                          h->d_own_in[2], h->d_own_in[3], h->d_own_in[4], h->d_own_in[5], s));
  for (int q = 0; q < 6; ++q) h->d_in[q] = h->d_own_in[q];
  h->d_flag = h->d_own_flag;
  h->d_u0 = h->d_own_u0;
  h->d_v0 = h->d_own_v0;
  h->d_w0 = h->d_own_w0;
  CKS(prepare_coefs(h));
  CK(cudaStreamSynchronize(s));
  h->have_inputs = true;
  return QESB_OK;
}

qesb_status qesb_set_inputs_device(qesb_handle *h, const float *e, const float *f, const float *g,
                                   const float *hc, const float *m, const float *n,
                                   const int *icellflag, const float *u0, const float *v0,
                                   const float *w0)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  if (!e || !f || !g || !hc || !m || !n || !icellflag || !u0 || !v0 || !w0)
    return qesb_fail(QESB_ERR_ARG, "qesb_set_inputs_device: null input");
  CK(cudaSetDevice(h->device));
  const float *src[6] = {e, f, g, hc, m, n};
  for (int q = 0; q < 6; ++q) h->d_in[q] = const_cast<float *>(src[q]);
  h->d_flag = const_cast<int *>(icellflag);
  h->d_u0 = const_cast<float *>(u0);
  h->d_v0 = const_cast<float *>(v0);
  h->d_w0 = const_cast<float *>(w0);
  CKS(prepare_coefs(h));
  CK(cudaStreamSynchronize(h->stream));
  h->have_inputs = true;
  return QESB_OK;
}

qesb_status qesb_wall_log_law(qesb_handle *h, float z0, float dz, float *u, float *v, float *w)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  if (!u || !v || !w) return qesb_fail(QESB_ERR_ARG, "qesb_wall_log_law: null wind array");
  if (!(z0 > 0.0f) || !(dz > 0.0f)) return qesb_fail(QESB_ERR_ARG, "qesb_wall_log_law: z0 and dz must be > 0");
  if (!h->have_inputs) return qesb_fail(QESB_ERR_STATE, "qesb_wall_log_law needs inputs (icellflag)");
  CK(cudaSetDevice(h->device));
  const DevGrid &G = h->G;
  cudaStream_t s = h->stream;
  if (!h->d_wbits) {
    CK(cudaMalloc((void **)&h->d_wbits, (size_t)G.XY * G.Z));
    CK(cudaMalloc((void **)&h->d_wcut, sizeof(int)));
  }
  CK(zero_async(h->d_wcut, sizeof(int), s));
  const dim3 grid((G.X + 127) / 128, G.Y, G.Z - 2), block(128);
  k_wall_bits<<<grid, block, 0, s>>>(G, h->d_flag, h->d_wbits, h->d_wcut);
  // the reference's distances: getDomainSize() is (dx, dx, dz) (Domain.h:104),
  // so the y walls use dx as well; its logarithms of floats are logf
  const float dxy = h->dx;
  const float lz21 = logf((1.5f * dz) / (0.5f * dz)), lz10 = logf((0.5f * dz) / z0);
  const float lx21 = logf((1.5f * dxy) / (0.5f * dxy)), lx10 = logf((0.5f * dxy) / z0);
  k_wall_log<kWallBelow><<<grid, block, 0, s>>>(G, h->d_wbits, h->d_wcut, u, v, w, lz21, lz10);
  k_wall_log<kWallAbove><<<grid, block, 0, s>>>(G, h->d_wbits, h->d_wcut, u, v, w, lz21, lz10);
  k_wall_log<kWallBack><<<grid, block, 0, s>>>(G, h->d_wbits, h->d_wcut, u, v, w, lx21, lx10);
  k_wall_log<kWallFront><<<grid, block, 0, s>>>(G, h->d_wbits, h->d_wcut, u, v, w, lx21, lx10);
  k_wall_log<kWallRight><<<grid, block, 0, s>>>(G, h->d_wbits, h->d_wcut, u, v, w, lx21, lx10);
  k_wall_log<kWallLeft><<<grid, block, 0, s>>>(G, h->d_wbits, h->d_wcut, u, v, w, lx21, lx10);
  CK(cudaGetLastError());
  int cut = 0;
  CK(cudaMemcpyAsync(&cut, h->d_wcut, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (cut)
    return qesb_fail(QESB_ERR_STATE,
                     "qesb_wall_log_law: cut-cell flags (7, 8) present; only stair-step walls are treated");
  return QESB_OK;
}

qesb_status qesb_solve_device(qesb_handle *h, int itermax, float *u, float *v, float *w, qesb_stats *st)
{
  return solve_impl(h, itermax, u, v, w, st);
}

qesb_status qesb_solve(qesb_handle *h, int itermax, float *u, float *v, float *w, qesb_stats *st)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  CK(cudaSetDevice(h->device));
  const size_t nf = (size_t)h->G.FXY * h->G.FZ;
  if (!h->d_u) {
    CKS(dalloc(&h->d_u, nf));
    CKS(dalloc(&h->d_v, nf));
    CKS(dalloc(&h->d_w, nf));
  }
  CKS(solve_impl(h, itermax, u ? h->d_u : nullptr, v ? h->d_v : nullptr, w ? h->d_w : nullptr, st));
  if (u) CK(cudaMemcpyAsync(u, h->d_u, nf * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  if (v) CK(cudaMemcpyAsync(v, h->d_v, nf * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  if (w) CK(cudaMemcpyAsync(w, h->d_w, nf * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return QESB_OK;
}

qesb_status qesb_set_lambda(qesb_handle *h, const float *lambda)
{
  if (!h || !lambda) return qesb_fail(QESB_ERR_ARG, "qesb_set_lambda: null argument");
  CK(cudaSetDevice(h->device));
  const DevGrid &G = h->G;
  const size_t nc = (size_t)G.XY * G.Z;
  float *tmp = nullptr;
  CKS(dalloc(&tmp, nc));
  cudaError_t e1 = cudaMemcpyAsync(tmp, lambda, nc * sizeof(float), cudaMemcpyHostToDevice, h->stream);
  if (e1 == cudaSuccess) {
    k_lambda_to_pad<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, h->stream>>>(G, tmp, h->d_lam);
    e1 = cudaGetLastError();
  }
  if (e1 == cudaSuccess) e1 = cudaStreamSynchronize(h->stream);
  cudaFree(tmp);
  if (e1 != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "qesb_set_lambda: %s", cudaGetErrorString(e1));
  return QESB_OK;
}

qesb_status qesb_get_lambda(qesb_handle *h, float *lambda)
{
  if (!h || !lambda) return qesb_fail(QESB_ERR_ARG, "qesb_get_lambda: null argument");
  CK(cudaSetDevice(h->device));
  const DevGrid &G = h->G;
  const size_t nc = (size_t)G.XY * G.Z;
  float *tmp = nullptr;
  CKS(dalloc(&tmp, nc));
  k_lambda_from_pad<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, h->stream>>>(G, h->d_lam, tmp);
  cudaError_t e1 = cudaGetLastError();
  if (e1 == cudaSuccess) e1 = cudaMemcpyAsync(lambda, tmp, nc * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
  if (e1 == cudaSuccess) e1 = cudaStreamSynchronize(h->stream);
  cudaFree(tmp);
  if (e1 != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "qesb_get_lambda: %s", cudaGetErrorString(e1));
  return QESB_OK;
}

qesb_status qesb_get_divergence(qesb_handle *h, float *R)
{
  if (!h || !R) return qesb_fail(QESB_ERR_ARG, "qesb_get_divergence: null argument");
  CK(cudaSetDevice(h->device));
  const DevGrid &G = h->G;
  const size_t nc = (size_t)G.XY * G.Z;
  float *tmp = nullptr;
  CKS(dalloc(&tmp, nc));
  k_lambda_from_pad<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, h->stream>>>(G, h->d_R, tmp);
  cudaError_t e1 = cudaGetLastError();
  if (e1 == cudaSuccess) e1 = cudaMemcpyAsync(R, tmp, nc * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
  if (e1 == cudaSuccess) e1 = cudaStreamSynchronize(h->stream);
  cudaFree(tmp);
  if (e1 != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "qesb_get_divergence: %s", cudaGetErrorString(e1));
  return QESB_OK;
}

qesb_status qesb_compute_divergence(qesb_handle *h)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  if (!h->have_inputs) return qesb_fail(QESB_ERR_STATE, "qesb_compute_divergence before qesb_set_inputs");
  CK(cudaSetDevice(h->device));
  const DevGrid &G = h->G;
  launch_divergence(h, h->stream);
  CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_warm_input(qesb_handle *h, void *x, int C, unsigned *scale)
{
  if (!h || !x || !scale || C < 8 || C % 8) return qesb_fail(QESB_ERR_ARG, "qesb_warm_input: bad arguments");
  CK(cudaSetDevice(h->device));
  const DevGrid &G = h->G;
  CK(zero_async(scale, sizeof(unsigned), h->stream));
  k_absmax_R<<<dim3((G.Y - 2 + 7) / 8, G.Z - 2), 256, 0, h->stream>>>(G, h->d_R, scale);
  double dzs = 0.0, height = 0.0;
  for (int k = 1; k < G.Z; ++k) dzs += h->dz[k];
  for (int k = 1; k < G.Z - 1; ++k) height += h->dz[k];
  k_warm_input<<<dim3((G.X + 127) / 128, G.Y, G.Z - 1), 128, 0, h->stream>>>(
      G, G.Z - 1, C, h->d_R, h->d_flag, h->d_dz, scale, (float)(dzs / (G.Z - 1)), (float)height, (uint16_t *)x);
  CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_warm_input_half(qesb_handle *h, void *x, int C, unsigned *scale)
{
  if (!h || !x || !scale || C < 8 || C % 8) return qesb_fail(QESB_ERR_ARG, "qesb_warm_input_half: bad arguments");
  const DevGrid &G = h->G;
  if (G.X % 2 || G.Y % 2 || (G.Z - 1) % 2)
    return qesb_fail(QESB_ERR_ARG, "qesb_warm_input_half: the net grid (Nz x Ny x Nx) must have even sizes");
  CK(cudaSetDevice(h->device));
  CK(zero_async(scale, sizeof(unsigned), h->stream));
  k_absmax_R<<<dim3((G.Y - 2 + 7) / 8, G.Z - 2), 256, 0, h->stream>>>(G, h->d_R, scale);
  double dzs = 0.0, height = 0.0;
  for (int k = 1; k < G.Z; ++k) dzs += h->dz[k];
  for (int k = 1; k < G.Z - 1; ++k) height += h->dz[k];
  k_warm_input_half<<<dim3((G.X / 2 + 127) / 128, G.Y / 2, (G.Z - 1) / 2), 128, 0, h->stream>>>(
      G, C, h->d_R, h->d_flag, h->d_dz, scale, (float)(dzs / (G.Z - 1)), (float)height, (uint16_t *)x);
  CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_warm_target(qesb_handle *h, float *tgt, float *w, const unsigned *scale)
{
  if (!h || !tgt || !w || !scale) return qesb_fail(QESB_ERR_ARG, "qesb_warm_target: bad arguments");
  CK(cudaSetDevice(h->device));
  k_warm_target<<<148 * 8, 256, 0, h->stream>>>(h->G, h->G.Z - 1, h->d_lam, scale, tgt, w);
  CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_warm_apply(qesb_handle *h, const float *yhead, int N, const unsigned *scale)
{
  if (!h || !yhead || !scale || N < 1) return qesb_fail(QESB_ERR_ARG, "qesb_warm_apply: bad arguments");
  CK(cudaSetDevice(h->device));
  k_warm_apply<<<dim3((h->G.X + 127) / 128, h->G.Y, h->G.Z), 128, 0, h->stream>>>(h->G, h->G.Z - 1, yhead, N,
                                                                                  scale, h->d_lam);
  CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_warm_apply_up2(qesb_handle *h, const float *yhead, int N, const unsigned *scale)
{
  if (!h || !yhead || !scale || N < 1) return qesb_fail(QESB_ERR_ARG, "qesb_warm_apply_up2: bad arguments");
  if ((h->G.Z - 1) % 2 || h->G.Y % 2 || h->G.X % 2)
    return qesb_fail(QESB_ERR_ARG, "qesb_warm_apply_up2: the net grid (Nz x Ny x Nx) must have even sizes");
  CK(cudaSetDevice(h->device));
  k_warm_apply_up2<<<dim3((h->G.X + 127) / 128, h->G.Y, h->G.Z), 128, 0, h->stream>>>(h->G, h->G.Z - 1, yhead, N,
                                                                                      scale, h->d_lam);
  CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_get_residual_history(qesb_handle *h, double *out, int n)
{
  if (!h || !out || n < 0) return qesb_fail(QESB_ERR_ARG, "qesb_get_residual_history: bad argument");
  if (n > h->err_cap) return qesb_fail(QESB_ERR_ARG, "qesb_get_residual_history: n exceeds the last solve");
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(out, h->d_err, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return QESB_OK;
}

qesb_status qesb_time_sweeps(qesb_handle *h, int n, float *ms, int *k)
{
  if (!h || n <= 0 || !ms) return qesb_fail(QESB_ERR_ARG, "qesb_time_sweeps: bad argument");
  if (!h->have_inputs || !h->packed) return qesb_fail(QESB_ERR_STATE, "qesb_time_sweeps needs stair-step inputs");
  CK(cudaSetDevice(h->device));
  if (pick_variant(h) >= kSplitVariant) {
    const SweepVariant &sv = kSweepVariants[pick_variant(h) - kSplitVariant];
    CKS(sweep_prepare(sv));
    CKS(ensure_err(h, n + 1));
    cudaStream_t s = h->stream;
    CK(zero_async(h->d_state, sizeof(SolveState), s));
    std::vector<SweepDomain> one{sweep_domain(h, 1 << 30, -1.0)};  // tol < 0: every launch runs
    CKS(attach_tmaps(h, sv, one[0], s));
    sweep_tiles(one, sv, false, h->device);
    CKS(h->list.upload(one, sv.unit, s));
    const dim3 grid(sweep_ctas(sv, false, h->device)), block(32, sv.block_y);
    SweepArgs a = h->list.a;
    a.one = one[0];
    a.wait_limit = h->opt_wait_limit;
    CK(cudaEventRecord(h->ev[0], s));
    for (int c = 0; c < n; ++c) {
      sv.red<<<grid, block, sv.smem, s>>>(a);
      sv.black<<<grid, block, sv.smem, s>>>(a);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(h->ev[1], s));
    CK(cudaEventSynchronize(h->ev[1]));
    CK(cudaEventElapsedTime(ms, h->ev[0], h->ev[1]));
    CK(cudaMemcpy(h->h_ctl, a.ctl, sizeof(SweepCtl), cudaMemcpyDeviceToHost));
    if (h->h_ctl->fault) return qesb_fail(QESB_ERR_CUDA, "sweep stage wait gave up");
    if (k) *k = 1;
    return QESB_OK;
  }
  const Variant &v = kVariants[pick_variant(h)];
  CKS(set_smem_attr(v));
  CKS(ensure_err(h, v.K));
  cudaStream_t s = h->stream;
  CK(zero_async(h->d_state, sizeof(SolveState), s));
  float *buf[2] = {h->d_lam, h->d_lam2};
  const dim3 grid = tiled_grid(h->G, v);
  CK(cudaEventRecord(h->ev[0], s));
  for (int c = 0; c < n; ++c)
    v.fn<<<grid, v.NT, v.smem, s>>>(tiled_args(h, buf[c & 1], buf[(c & 1) ^ 1], 1 << 30, 0));
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev[1], s));
  CK(cudaEventSynchronize(h->ev[1]));
  CK(cudaEventElapsedTime(ms, h->ev[0], h->ev[1]));
  if (n & 1) std::swap(h->d_lam, h->d_lam2);
  if (k) *k = v.K;
  return QESB_OK;
}

int qesb_num_variants(void) { return kAllVariants; }

qesb_status qesb_autotune(qesb_handle *h, int *best, float *us_per_iter, int n_variants)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  if (!h->have_inputs || !h->packed) return qesb_fail(QESB_ERR_STATE, "qesb_autotune needs stair-step inputs");
  CK(cudaSetDevice(h->device));
  const int nv = kAllVariants;
  const size_t np = pad_alloc(h->G);
  float *saved = nullptr;
  CKS(dalloc(&saved, np));
  cudaStream_t s = h->stream;
  CK(cudaMemcpyAsync(saved, h->d_lam, np * sizeof(float), cudaMemcpyDeviceToDevice, s));
  const int keep = h->opt_variant;
  int arg = -1;
  float best_us = 0.0f;
  qesb_status st = QESB_OK;
  for (int v = 0; v < nv && st == QESB_OK; ++v) {
    h->opt_variant = v;
    float ms = 0.0f;
    int k = 1;
    st = qesb_time_sweeps(h, 2, &ms, &k);  // warm-up
    if (st != QESB_OK) break;
    st = qesb_time_sweeps(h, 2, &ms, &k);
    if (st != QESB_OK) break;
    const int n = std::max(2, std::min(64, (int)(8.0f / std::max(ms / 2, 1e-3f))));
    st = qesb_time_sweeps(h, n, &ms, &k);
    if (st != QESB_OK) break;
    const float us = 1000.0f * ms / (n * k);
    if (us_per_iter && v < n_variants) us_per_iter[v] = us;
    if (arg < 0 || us < best_us) {
      arg = v;
      best_us = us;
    }
  }
  h->opt_variant = keep;
  cudaMemcpyAsync(h->d_lam, saved, np * sizeof(float), cudaMemcpyDeviceToDevice, s);
  cudaStreamSynchronize(s);
  cudaFree(saved);
  if (st != QESB_OK) return st;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[{h->G.X, h->G.Y, h->G.Z}] = arg;
  }
  if (best) *best = arg;
  return QESB_OK;
}

// Checks shared by the batch entry points.
static qesb_status batch_check(qesb_handle *const *hs, int n, const char *who)
{
  if (!hs || n <= 0) return qesb_fail(QESB_ERR_ARG, "%s: bad argument", who);
  for (int i = 0; i < n; ++i) {
    if (!hs[i]) return qesb_fail(QESB_ERR_ARG, "%s: null handle %d", who, i);
    if (!hs[i]->have_inputs) return qesb_fail(QESB_ERR_STATE, "%s: domain %d has no inputs", who, i);
    if (!hs[i]->packed || hs[i]->opt_path != 1)
      return qesb_fail(QESB_ERR_STATE, "%s: domain %d is not on the packed (stair-step) path", who, i);
    if (hs[i]->device != hs[0]->device) return qesb_fail(QESB_ERR_ARG, "%s: handles on two devices", who);
    for (int k = 0; k < i; ++k)
      if (hs[k] == hs[i]) return qesb_fail(QESB_ERR_ARG, "%s: handle %d repeated", who, i);
  }
  return QESB_OK;
}

qesb_status qesb_autotune_batch(qesb_handle *const *hs, int n, int *best, float *us_per_iter, int n_variants)
{
  CKS(batch_check(hs, n, "qesb_autotune_batch"));
  qesb_handle *h0 = hs[0];
  CK(cudaSetDevice(h0->device));
  cudaStream_t s = h0->stream;
  // the domains as a solve would start them: R, and lambda and R in the split
  // layout (the tuning sweeps advance only the split copy; a solve re-derives
  // it from lambda)
  for (int i = 0; i < n; ++i) {
    qesb_handle *h = hs[i];
    const DevGrid &G = h->G;
    launch_divergence(h, s);
    k_pad_to_split<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, s>>>(G, h->S, h->d_lam, h->d_lam_s);
    k_pad_to_split<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, s>>>(G, h->S, h->d_R, h->d_R_s);
  }
  CK(cudaGetLastError());
  SweepList list;
  CKS(list.create(n));
  qesb_status qs = QESB_OK;
  int arg = -1;
  float best_us = 0.0f;
  for (int v = kSplitVariant; v < kAllVariants && qs == QESB_OK; ++v) {
    const SweepVariant &sv = kSweepVariants[v - kSplitVariant];
    qs = sweep_prepare(sv);
    const dim3 grid(sweep_ctas(sv, true, h0->device)), block(32, sv.block_y);
    float ms = 0.0f;
    int reps = 2;
    for (int pass = 0; pass < 3 && qs == QESB_OK; ++pass) {
      // pass 0 warms up, pass 1 sizes the timed pass 2 to about 8 ms
      std::vector<SweepDomain> doms(n);
      for (int i = 0; i < n && qs == QESB_OK; ++i) {
        qs = ensure_err(hs[i], reps + 1);
        if (qs != QESB_OK) break;
        if (zero_async(hs[i]->d_err, sizeof(double) * (reps + 1), s) != cudaSuccess ||
            zero_async(hs[i]->d_state, sizeof(SolveState), s) != cudaSuccess)
          qs = qesb_fail(QESB_ERR_CUDA, "qesb_autotune_batch: memset");
        doms[i] = sweep_domain(hs[i], 1 << 30, -1.0);  // tol < 0: every launch runs
        if (qs == QESB_OK) qs = attach_tmaps(hs[i], sv, doms[i], s);
      }
      if (qs != QESB_OK) break;
      sweep_tiles(doms, sv, true, h0->device);
      qs = list.upload(doms, sv.unit, s);
      if (qs != QESB_OK) break;
      cudaEventRecord(h0->ev[0], s);
      for (int c = 0; c < reps; ++c) {
        sv.red_m<<<grid, block, sv.smem, s>>>(list.a);
        sv.black_m<<<grid, block, sv.smem, s>>>(list.a);
      }
      cudaEventRecord(h0->ev[1], s);
      if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(h0->ev[1]) != cudaSuccess ||
          cudaEventElapsedTime(&ms, h0->ev[0], h0->ev[1]) != cudaSuccess) {
        qs = qesb_fail(QESB_ERR_CUDA, "qesb_autotune_batch: variant %d launch failed", v);
        break;
      }
      SweepCtl ctl;
      if (cudaMemcpy(&ctl, list.a.ctl, sizeof ctl, cudaMemcpyDeviceToHost) != cudaSuccess || ctl.fault) {
        qs = qesb_fail(QESB_ERR_CUDA, "qesb_autotune_batch: variant %d stage wait gave up", v);
        break;
      }
      if (pass == 1) reps = std::max(2, std::min(64, (int)(8.0f / std::max(ms / reps, 1e-3f))));
    }
    if (qs != QESB_OK) break;
    const float us = 1000.0f * ms / reps;
    if (us_per_iter && v < n_variants) us_per_iter[v] = us;
    if (arg < 0 || us < best_us) {
      arg = v;
      best_us = us;
    }
  }
  list.destroy();
  if (qs != QESB_OK) return qs;
  h0->opt_batch_variant = arg;
  if (best) *best = arg;
  return QESB_OK;
}

qesb_status qesb_solve_batch(qesb_handle *const *hs, int n, int itermax, float *const *u, float *const *v,
                             float *const *w, qesb_stats *st)
{
  if (itermax < 0) return qesb_fail(QESB_ERR_ARG, "qesb_solve_batch: bad argument");
  CKS(batch_check(hs, n, "qesb_solve_batch"));
  qesb_handle *h0 = hs[0];
  CK(cudaSetDevice(h0->device));
  cudaStream_t s = h0->stream;
  // launch shape: handles[0]'s "batch_variant" option (qesb_autotune_batch),
  // else its "variant" option when it names a sweep shape, else its grid's
  // autotuned shape when that is one, else the default
  int vi = h0->opt_batch_variant >= kSplitVariant ? h0->opt_batch_variant
           : h0->opt_variant >= kSplitVariant    ? h0->opt_variant
                                                 : tuned_variant(h0->G);
  if (vi < kSplitVariant) vi = kSplitVariant + kDefaultSweep;
  const SweepVariant &sv = kSweepVariants[vi - kSplitVariant];
  CK(cudaEventRecord(h0->ev[0], s));
  std::vector<SweepDomain> doms(n);
  double cells = 0;
  std::vector<SweepDomain> pre, start;
  std::vector<int> pre_of, start_of;  // batch index of each pre-phase / start-stage domain
  for (int i = 1; i < n; ++i)
    if (hs[i]->win_k != h0->win_k)
      return qesb_fail(QESB_ERR_ARG, "qesb_solve_batch: handles %d and 0 have different window lengths (%d, %d)", i,
                       hs[i]->win_k, h0->win_k);
  WordBatch wb(s);  // the domains' small fills and state reads, one launch per group
  for (int i = 0; i < n; ++i) {
    qesb_handle *h = hs[i];
    const DevGrid &G = h->G;
    const bool pre_on = prephase_on(h) && itermax > 0;
    const int nerr = err_slots(h, itermax);
    CKS(ensure_err(h, nerr));
    ensure_divergence(h, s);
    CKS(wb.zero(h->d_err, sizeof(double) * nerr));
    h->last_pre_iterations = 0;
    if (pre_on) {
      SweepDomain p;
      CKS(sweep_domain_pre(h, p, s));
      CKS(attach_tmaps(h, sv, p, s));
      pre.push_back(p);
      pre_of.push_back(i);
      if (start_on(h)) {
        CKS(sweep_domain_start(h, p, s));
        CKS(attach_tmaps(h, sv, p, s));
        start.push_back(p);
        start_of.push_back(i);
      }
    }
    CKS(wb.zero(h->d_state, sizeof(SolveState)));
    k_pad_to_split<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, s>>>(G, h->S, h->d_lam, h->d_lam_s);
    k_pad_to_split<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, s>>>(G, h->S, h->d_R, h->d_R_s);
    CK(cudaGetLastError());
    doms[i] = sweep_domain(h, itermax, (double)h->tol);
    CKS(attach_tmaps(h, sv, doms[i], s));
    cells += (double)G.XY * G.Z;
  }
  CKS(wb.flush());
  SweepList &list = h0->blist;
  if (list.cap < n) {
    list.destroy();
    CKS(list.create(n));
  }
  list.a.wait_limit = h0->opt_wait_limit;
  k_sweep_stamp<<<1, 1, 0, s>>>(list.a.ctl);  // the latencies (ms_sor) count from here
  qesb_status qs = QESB_OK;
  int launched = 0, pre_launched = 0;
  CK(cudaEventRecord(h0->evs[0], s));
  if (!start.empty()) {
    // the start stages of the pre-phases that have one, as a list of their own
    sweep_tiles(start, sv, true, h0->device);
    qs = list.upload(start, sv.unit, s);
    int smax = 0;
    for (int i : start_of) smax = std::max(smax, hs[i]->start_iters);
    int n1 = 0;
    if (qs == QESB_OK)
      qs = run_sweep_loop(sv, true, list.a, h0->device, s, cells, smax, h0->opt_graph != 0, &h0->bgraph_start,
                          h0->h_ctl, h0->h_ctl_dev, &n1, 0, 1, h0->opt_pdl != 0);
    pre_launched += n1;
    for (size_t q = 0; q < start_of.size() && qs == QESB_OK; ++q)
      qs = wb.add(hs[start_of[q]]->h_state_dev, hs[start_of[q]]->d_state, sizeof(SolveState));
    if (qs == QESB_OK) qs = wb.flush();
    if (qs == QESB_OK) CK(cudaStreamSynchronize(s));
    for (size_t q = 0; q < start_of.size() && qs == QESB_OK; ++q) {
      qesb_handle *h = hs[start_of[q]];
      const SolveState sp = *h->h_state;
      if (sp.nan)
        qs = qesb_fail(QESB_ERR_NUMERIC, "NaN in lambda of batch domain %d during the pre-phase's start stage",
                       start_of[q]);
      h->last_pre_iterations = sp.it;
      if (qs == QESB_OK) qs = wb.zero(h->d_err, sizeof(double) * err_slots(h, itermax));
      if (qs == QESB_OK) qs = wb.zero(h->d_state, sizeof(SolveState));
    }
    if (qs == QESB_OK) qs = wb.flush();
  }
  if (!pre.empty() && qs == QESB_OK) {
    // the over-relaxed pre-phase of the domains that have one, as a list of its own
    sweep_tiles(pre, sv, true, h0->device);
    qs = list.upload(pre, sv.unit, s);
    int pre_max = 0;
    for (int i : pre_of) pre_max = std::max(pre_max, hs[i]->pre_iters);
    int n2 = 0;
    if (qs == QESB_OK)
      qs = run_sweep_loop(sv, true, list.a, h0->device, s, cells, pre_max, h0->opt_graph != 0, &h0->bgraph_pre,
                          h0->h_ctl, h0->h_ctl_dev, &n2, 0, 1, h0->opt_pdl != 0);
    pre_launched += n2;
    for (size_t q = 0; q < pre_of.size() && qs == QESB_OK; ++q)
      qs = wb.add(hs[pre_of[q]]->h_state_dev, hs[pre_of[q]]->d_state, sizeof(SolveState));
    if (qs == QESB_OK) qs = wb.flush();
    if (qs == QESB_OK) CK(cudaStreamSynchronize(s));
    for (size_t q = 0; q < pre_of.size() && qs == QESB_OK; ++q) {
      qesb_handle *h = hs[pre_of[q]];
      const SolveState sp = *h->h_state;
      if (sp.nan) qs = qesb_fail(QESB_ERR_NUMERIC, "NaN in lambda of batch domain %d during the pre-phase", pre_of[q]);
      h->last_pre_iterations += sp.it;
      if (qs == QESB_OK) qs = wb.zero(h->d_err, sizeof(double) * std::max(itermax, 1));
      if (qs == QESB_OK) qs = wb.zero(h->d_state, sizeof(SolveState));
    }
    if (qs == QESB_OK) qs = wb.flush();
  }
  CK(cudaEventRecord(h0->evs[1], s));
  sweep_tiles(doms, sv, true, h0->device);
  if (qs == QESB_OK) qs = list.upload(doms, sv.unit, s);
  if (qs == QESB_OK && h0->win_k > 0)  // each domain's first window starts from lambda as the loop begins
    for (int i = 0; i < n && qs == QESB_OK; ++i)
      qs = copy_floats(hs[i]->d_snap, hs[i]->d_lam_s, 2L * hs[i]->S.CS, s);
  if (qs == QESB_OK) {
    CK(cudaEventRecord(h0->evs[2], s));
    if (itermax > 0)
      qs = run_sweep_loop(sv, true, list.a, h0->device, s, cells, itermax, h0->opt_graph != 0, &h0->bgraph, h0->h_ctl,
                          h0->h_ctl_dev, &launched, h0->win_k, n, h0->opt_pdl != 0);
    CK(cudaEventRecord(h0->evs[3], s));
  }
  const unsigned long long t0 = h0->h_ctl->t0;
  CK(cudaEventRecord(h0->ev[2], s));
  for (int i = 0; i < n && qs == QESB_OK; ++i) {
    qesb_handle *h = hs[i];
    const DevGrid &G = h->G;
    k_split_mirror_ring<<<G.Y, 128, 0, s>>>(G, h->S, h->d_lam_s);
    k_split_to_pad<<<row_grid(G, G.Y, G.Z, G.X), 256, 0, s>>>(G, h->S, h->d_lam_s, h->d_lam);
    k_correct<<<dim3(1, (G.FY + 7) / 8, G.FZ), dim3(32, 8), 0, s>>>(
        G, h->d_lam, h->d_in[1], h->d_in[3], h->d_in[5], h->d_flag, h->d_u0, h->d_v0, h->d_w0, h->d_dz, h->dx,
        h->dy, u ? u[i] : nullptr, v ? v[i] : nullptr, w ? w[i] : nullptr);
    cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) qs = qesb_fail(QESB_ERR_CUDA, "batch finish: %s", cudaGetErrorString(ce));
    if (qs == QESB_OK && u && v && w && u[i] && v[i] && w[i]) qs = enqueue_divergence_check(h, u[i], v[i], w[i], s);
  }
  CK(cudaEventRecord(h0->ev[3], s));
  // every domain's final state and divergence into its mapped buffers, then one wait
  for (int i = 0; i < n && qs == QESB_OK; ++i) {
    qs = wb.add(hs[i]->h_state_dev, hs[i]->d_state, sizeof(SolveState));
    if (qs == QESB_OK) qs = wb.add(hs[i]->h_io_dev, hs[i]->d_div, sizeof(double));
  }
  if (qs == QESB_OK) qs = wb.flush();
  cudaError_t se = cudaStreamSynchronize(s);
  if (qs != QESB_OK) return qs;
  if (se != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "batch: %s", cudaGetErrorString(se));
  float ms_all = 0, ms_pre = 0, ms_ref = 0;
  CK(cudaEventElapsedTime(&ms_all, h0->ev[0], h0->ev[3]));
  CK(cudaEventElapsedTime(&ms_pre, h0->evs[0], h0->evs[1]));
  CK(cudaEventElapsedTime(&ms_ref, h0->evs[2], h0->evs[3]));
  int nan_at = -1;
  for (int i = 0; i < n; ++i) {
    const SolveState sti = *hs[i]->h_state;
    double div = -1.0;
    if (u && v && w && u[i] && v[i] && w[i]) std::memcpy(&div, hs[i]->h_io, sizeof div);
    if (st) st[i].max_divergence = div;
    if (sti.nan && nan_at < 0) nan_at = i;
    if (st) {
      st[i].iterations = itermax > 0 ? sti.it : 0;
      st[i].converged = sti.converged;
      st[i].residual = itermax > 0 ? sti.residual : 1.0;
      st[i].ms_total = ms_all;
      st[i].ms_sor = sti.t_done > t0 ? (double)(sti.t_done - t0) * 1e-6 : 0.0;
      st[i].path = 1;
      st[i].sweeps_per_launch = 1;
      st[i].launches = 2 * (launched + pre_launched) + (h0->win_k > 0 ? launched / h0->win_k : 0);
      st[i].pre_iterations = hs[i]->last_pre_iterations;
      st[i].window_drift = h0->win_k > 0 && st[i].iterations >= h0->win_k ? sti.wdrift : -1.0;
      st[i].ms_sweeps = (double)ms_pre + (double)ms_ref;
    }
  }
  if (nan_at >= 0) return qesb_fail(QESB_ERR_NUMERIC, "NaN in lambda of batch domain %d", nan_at);
  return QESB_OK;
}

qesb_status qesb_set_prephase_start(qesb_handle *h, float omega, int iterations)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  if (iterations < 0 || (iterations > 0 && !(omega > 0.0f && omega < 2.0f)))
    return qesb_fail(QESB_ERR_ARG, "qesb_set_prephase_start: iterations must be >= 0 and omega in (0, 2)");
  h->start_omega = iterations > 0 ? omega : 0.0f;
  h->start_iters = iterations;
  return QESB_OK;
}

qesb_status qesb_set_prephase(qesb_handle *h, float omega, float tol, int max_iterations)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  if (omega != 0.0f && !(omega > 1.0f && omega < 2.0f))
    return qesb_fail(QESB_ERR_ARG, "qesb_set_prephase: omega must be 0 (off) or in (1, 2)");
  if (max_iterations < 0) return qesb_fail(QESB_ERR_ARG, "qesb_set_prephase: max_iterations must be >= 0");
  h->pre_omega = omega;
  h->pre_tol = tol;
  h->pre_iters = max_iterations;
  return QESB_OK;
}

}  // extern "C"

qesb_status qesb_handle_grid(qesb_handle *h, int *Nx, int *Ny, int *Nz, int *device)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  *Nx = h->G.X;
  *Ny = h->G.Y;
  *Nz = h->G.Z - 1;
  *device = h->device;
  return QESB_OK;
}

extern "C" {

qesb_status qesb_fp64_same_sor(qesb_handle *h, const float *lambda0, float pre_omega, int pre_iterations,
                               int iterations, const float *u, const float *v, const float *w, double *lambda64,
                               qesb_fp64_report *rep)
{
  if (!h || !rep || pre_iterations < 0 || iterations < 0 || (pre_iterations > 0 && !(pre_omega > 0.0f)))
    return qesb_fail(QESB_ERR_ARG, "qesb_fp64_same_sor: bad argument");
  if (!h->have_inputs) return qesb_fail(QESB_ERR_STATE, "qesb_fp64_same_sor before qesb_set_inputs");
  CK(cudaSetDevice(h->device));
  const DevGrid &G = h->G;
  cudaStream_t s = h->stream;
  const size_t nc = (size_t)G.XY * G.Z;
  double *L = nullptr, *R = nullptr, *acc = nullptr;
  auto release = [&]() {
    cudaFree(L);
    cudaFree(R);
    cudaFree(acc);
  };
  if (dalloc(&L, nc) != QESB_OK || dalloc(&R, nc) != QESB_OK || dalloc(&acc, 4) != QESB_OK) {
    release();
    return qesb_fail(QESB_ERR_NOMEM, "qesb_fp64_same_sor: no room for the FP64 lambda and R");
  }
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
    return e == cudaSuccess;
  };
  if (lambda0) {  // the start, widened to double (R's buffer holds the floats meanwhile)
    float *tmp = reinterpret_cast<float *>(R);
    ok(cudaMemcpyAsync(tmp, lambda0, nc * sizeof(float), cudaMemcpyHostToDevice, s));
    k_widen64<<<(unsigned)((nc + 255) / 256), 256, 0, s>>>(tmp, L, (long)nc);
  } else {
    ok(zero_async(L, nc * sizeof(double), s));
  }
  ok(zero_async(R, nc * sizeof(double), s));
  ok(zero_async(acc, 4 * sizeof(double), s));
  ok(cudaEventRecord(h->ev[0], s));
  k_div64<<<row_grid(G, G.Y, G.Z - 2, G.X), 256, 0, s>>>(G, h->d_in[0], h->d_in[1], h->d_in[2], h->d_in[3],
                                                          h->d_in[4], h->d_in[5], h->d_u0, h->d_v0, h->d_w0,
                                                          h->d_dz, h->dx, h->dy, R);
  const dim3 sgrid(((G.X - 2) / 2 + 1 + 127) / 128, G.Y - 2, G.Z - 2), mgrid((G.X + 255) / 256, G.Y, 1);
  // phases: the handle's start stage (its share of pre_iterations), the rest
  // of the pre-phase at pre_omega, the reference loop
  const int n_start = start_on(h) ? std::min(h->start_iters, pre_iterations) : 0;
  for (int phase = 0; phase < 3 && e == cudaSuccess; ++phase) {
    const int n = phase == 0 ? n_start : phase == 1 ? pre_iterations - n_start : iterations;
    const double om = phase == 0 ? (double)h->start_omega : phase == 1 ? (double)pre_omega : (double)kOmega;
    for (int t = 0; t < n; ++t) {
      for (int colour = 0; colour < 2; ++colour)
        k_sor64<<<sgrid, 128, 0, s>>>(G, colour, om, h->d_in[0], h->d_in[1], h->d_in[2], h->d_in[3], h->d_in[4],
                                      h->d_in[5], R, L);
      k_mirror64<<<mgrid, 256, 0, s>>>(G, L);
      if ((t & 255) == 255 && !ok(cudaGetLastError())) break;
    }
  }
  ok(cudaGetLastError());
  ok(cudaEventRecord(h->ev[1], s));
  k_lambda_cmp64<<<dim3((G.X + 255) / 256, G.Y, G.Z), 256, 0, s>>>(G, L, h->d_lam, acc);
  const bool winds = u && v && w;
  if (winds)
    k_correct_cmp64<<<dim3((G.FX + 255) / 256, G.FY, G.FZ), 256, 0, s>>>(
        G, L, h->d_in[1], h->d_in[3], h->d_in[5], h->d_flag, h->d_u0, h->d_v0, h->d_w0, h->d_dz, h->dx, h->dy, u,
        v, w, acc + 2);
  ok(cudaGetLastError());
  double host[4] = {0, 0, 0, 0};
  ok(cudaMemcpyAsync(host, acc, sizeof host, cudaMemcpyDeviceToHost, s));
  if (lambda64) ok(cudaMemcpyAsync(lambda64, L, nc * sizeof(double), cudaMemcpyDeviceToHost, s));
  ok(cudaStreamSynchronize(s));
  float ms = 0.0f;
  if (e == cudaSuccess) ok(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
  release();
  if (e != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "qesb_fp64_same_sor: %s", cudaGetErrorString(e));
  rep->lambda_max_abs_err = host[0];
  rep->lambda_max_abs = host[1];
  rep->wind_max_err = winds ? host[2] : -1.0;
  rep->ms = ms;
  return QESB_OK;
}

qesb_status qesb_set_window_rule(qesb_handle *h, int window, double tol)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  if (window < 0 || window > 4096 || (window > 0 && !(tol >= 0.0)))
    return qesb_fail(QESB_ERR_ARG, "qesb_set_window_rule: window must be in [0, 4096] and tol >= 0");
  if (window > 0 && !h->d_snap) {
    CK(cudaSetDevice(h->device));
    const size_t nsnap = std::max((size_t)(2 * h->S.CS), pad_cells(h->G));
    CKS(dalloc(&h->d_snap, nsnap));
  }
  h->win_k = window;
  h->win_tol = tol;
  return QESB_OK;
}

qesb_status qesb_set_tolerance(qesb_handle *h, float tol)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  h->tol = tol;
  return QESB_OK;
}

qesb_status qesb_set_option(qesb_handle *h, const char *key, int value)
{
  if (!h || !key) return qesb_fail(QESB_ERR_ARG, "qesb_set_option: null argument");
  std::string k(key);
  if (k == "sweeps_per_launch") {
    if (value < 0 || value > 2) return qesb_fail(QESB_ERR_ARG, "sweeps_per_launch must be 0 (auto), 1 or 2");
    h->opt_k = value;
  } else if (k == "path") {
    if (value != 0 && value != 1) return qesb_fail(QESB_ERR_ARG, "path must be 0 or 1");
    h->opt_path = value;
  } else if (k == "graph") {
    h->opt_graph = value ? 1 : 0;
  } else if (k == "pdl") {
    h->opt_pdl = value ? 1 : 0;
  } else if (k == "autotune") {
    h->opt_autotune = value ? 1 : 0;
  } else if (k == "variant") {
    if (value < -1 || value >= kAllVariants)
      return qesb_fail(QESB_ERR_ARG, "variant must be in [-1, %d)", kAllVariants);
    h->opt_variant = value;
  } else if (k == "wait_limit") {
    if (value < 0) return qesb_fail(QESB_ERR_ARG, "wait_limit must be >= 0 (0: the default)");
    h->opt_wait_limit = (unsigned)value;
  } else if (k == "batch_variant") {
    if (value != -1 && (value < kSplitVariant || value >= kAllVariants))
      return qesb_fail(QESB_ERR_ARG, "batch_variant must be -1 or a sweep variant in [%d, %d)", kSplitVariant,
                       kAllVariants);
    h->opt_batch_variant = value;
  } else {
    return qesb_fail(QESB_ERR_ARG, "unknown option '%s'", key);
  }
  return QESB_OK;
}

qesb_status qesb_set_stream(qesb_handle *h, void *stream)
{
  if (!h) return qesb_fail(QESB_ERR_ARG, "null handle");
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return QESB_OK;
}

qesb_status qesb_get_stream(qesb_handle *h, void **stream)
{
  if (!h || !stream) return qesb_fail(QESB_ERR_ARG, "qesb_get_stream: null argument");
  *stream = h->stream;
  return QESB_OK;
}

}  // extern "C"
