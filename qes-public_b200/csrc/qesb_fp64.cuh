// FP64 run of the same red-black SOR, on the device: the precision check of
// an FP32 solve (qesb_fp64_same_sor). Included by qesb_solver.cu, so compiled
// with -fmad=false: every product and sum rounds as written, in double, in
// the order of the FP64 restatement the tests pin it to (R with each product
// formed in double, Solver_CPU.cpp:56-77; the SOR update of
// Solver_CPU_RB.cpp:118-125 with omega and the coefficient sum in double; the
// correction of Solver_CPU.cpp:157-231). Arrays in the reference cell and
// face layouts; lambda and R in double.
#pragma once
#include "qesb_device.cuh"

namespace qesb {

__global__ void k_div64(DevGrid G, const float *__restrict__ e, const float *__restrict__ f,
                        const float *__restrict__ g, const float *__restrict__ h, const float *__restrict__ m,
                        const float *__restrict__ n, const float *__restrict__ u0, const float *__restrict__ v0,
                        const float *__restrict__ w0, const float *__restrict__ dz, float dx, float dy,
                        double *__restrict__ R)
{
  const int j = blockIdx.y, k = blockIdx.z + 1;  // k in [1, nz-3]
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x) {
    const long c = G.cell(i, j, k), fc = G.face(i, j, k);
    const double xt = ((double)e[c] * u0[fc + 1] - (double)f[c] * u0[fc]) * dx;
    const double yt = ((double)g[c] * v0[fc + G.FX] - (double)h[c] * v0[fc]) * dy;
    const double zt = (double)m[c] * dz[k] * 0.5 * ((double)dz[k] + dz[k + 1]) * w0[fc + G.FXY] -
                      (double)n[c] * dz[k] * 0.5 * ((double)dz[k] + dz[k - 1]) * w0[fc];
    R[c] = -2.0 * (xt + yt + zt);
  }
}

// One colour of the sweep: cells with (i + j + k) % 2 == colour, i, j, k in
// [1, n-3] (the reference's loop bounds).
__global__ void __launch_bounds__(128) k_sor64(DevGrid G, int colour, double om, const float *__restrict__ pe,
                                               const float *__restrict__ pf, const float *__restrict__ pg,
                                               const float *__restrict__ ph, const float *__restrict__ pm,
                                               const float *__restrict__ pn, const double *__restrict__ R,
                                               double *__restrict__ L)
{
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  const int o = (colour + 1 + j + k) & 1;
  const int i = 1 + 2 * (int)(blockIdx.x * blockDim.x + threadIdx.x) + o;
  if (i > G.X - 2) return;
  const long c = G.cell(i, j, k);
  const float e = pe[c], f = pf[c], g = pg[c], h = ph[c], m = pm[c], n = pn[c];
  const double s = (double)e + f + g + h + m + n;
  L[c] = om / s *
             ((double)e * L[c + 1] + (double)f * L[c - 1] + (double)g * L[c + G.X] + (double)h * L[c - G.X] +
              (double)m * L[c + G.XY] + (double)n * L[c - G.XY] - R[c]) +
         (1.0 - om) * L[c];
}

__global__ void k_widen64(const float *__restrict__ x, double *__restrict__ y, long n)
{
  const long i = threadIdx.x + (long)blockIdx.x * blockDim.x;
  if (i < n) y[i] = x[i];
}

__global__ void k_mirror64(DevGrid G, double *__restrict__ L)
{
  const int j = blockIdx.y;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x)
    L[G.cell(i, j, 0)] = L[G.cell(i, j, 1)];
}

// max |L32 - L64| and max |L64| over all cells into out[0], out[1]
// (non-negative doubles: atomicMax on their bits). L32 in the padded layout.
__global__ void k_lambda_cmp64(DevGrid G, const double *__restrict__ L64, const float *__restrict__ L32,
                               double *out)
{
  const int j = blockIdx.y, k = blockIdx.z;
  double d = 0.0, a = 0.0;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x) {
    const double x = L64[G.cell(i, j, k)];
    const double dd = fabs((double)L32[G.pad(i, j, k)] - x), ax = fabs(x);
    if (dd > d || dd != dd) d = dd;
    if (ax > a || ax != ax) a = ax;
  }
  block_max_to(out, d);
  __syncthreads();  // both folds use block_max_to's one shared scratch array
  block_max_to(out + 1, a);
}

// The correction and solid-face zeroing in double (as k_correct), each face's
// value compared with the FP32 winds: max |x32 - x64| over u, v, w into *out.
__global__ void k_correct_cmp64(DevGrid G, const double *__restrict__ L, const float *__restrict__ f,
                                const float *__restrict__ h, const float *__restrict__ n,
                                const int *__restrict__ flag, const float *__restrict__ u0,
                                const float *__restrict__ v0, const float *__restrict__ w0,
                                const float *__restrict__ dz, float dx, float dy, const float *__restrict__ u,
                                const float *__restrict__ v, const float *__restrict__ w, double *out)
{
  const int j = blockIdx.y, k = blockIdx.z;
  double dmax = 0.0;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.FX; i += gridDim.x * blockDim.x) {
    const long q = G.face(i, j, k);
    double uu = u0[q], vv = v0[q], ww = w0[q];
    if (i >= 1 && i <= G.FX - 2 && j >= 1 && j <= G.FY - 2 && k >= 1 && k <= G.FZ - 3) {
      const long c = G.cell(i, j, k);
      uu = u0[q] + 0.5 * f[c] * dx * (L[c] - L[c - 1]);
      vv = v0[q] + 0.5 * h[c] * dy * (L[c] - L[c - G.X]);
      ww = w0[q] + 0.5 * n[c] * dz[k] * (L[c] - L[c - G.XY]);
    }
    const bool kin = k >= 1 && k <= G.FZ - 2;
    const bool ic = i <= G.X - 1, jc = j <= G.Y - 1;
    if (kin && jc && ((ic && is_solid(flag[G.cell(i, j, k)])) || (i >= 1 && is_solid(flag[G.cell(i - 1, j, k)]))))
      uu = 0.0;
    if (kin && ic && ((jc && is_solid(flag[G.cell(i, j, k)])) || (j >= 1 && is_solid(flag[G.cell(i, j - 1, k)]))))
      vv = 0.0;
    if (ic && jc && ((kin && is_solid(flag[G.cell(i, j, k)])) ||
                     (k - 1 >= 1 && k - 1 <= G.FZ - 2 && is_solid(flag[G.cell(i, j, k - 1)]))))
      ww = 0.0;
    const double d[3] = {fabs((double)u[q] - uu), fabs((double)v[q] - vv), fabs((double)w[q] - ww)};
#pragma unroll
    for (int t = 0; t < 3; ++t)
      if (d[t] > dmax || d[t] != d[t]) dmax = d[t];
  }
  block_max_to(out, dmax);
}

}  // namespace qesb
