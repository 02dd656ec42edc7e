// Red/black split-layout SOR half-sweeps (the packed path's streaming kernels).
// Included by qesb_solver.cu, so compiled with -fmad=false: each update rounds
// exactly as Solver_CPU_RB.cpp:118-125 does.
//
// Layout. Each cell field of the sweep (lambda, R, wall mask) is stored as two
// colour arrays. Colour c = (i + j + k) % 2 holds, for every row (j, k), the
// cells of that colour in x order: cell (i, j, k) sits at
//     sidx(c, i >> 1, j, k) = c*CS + (k*Y + j)*PQ + (i >> 1),
// PQ = roundup((X + 1) / 2, 32) (128-byte rows), CS = PQ*Y*Z. A half-sweep
// of colour c reads its own cells and the other colour's six neighbours:
//     x-1 -> (1-c, q - 1 + i0, j, k),  x+1 -> (1-c, q + i0, j, k),
//     y+-1 -> (1-c, q, j+-1, k),       z+-1 -> (1-c, q, j, k+-1),
// with i0 = (c + j + k) & 1 the x parity of the row's colour-c cells. A warp
// therefore loads 32 consecutive words for every operand, and each byte of
// the other colour is fetched from DRAM about once per half-sweep.
//
// Iteration = red kernel (colour 0) + black kernel (colour 1). The black
// kernel also applies the ground mirror lambda(k=0) <- lambda(k=1) to interior
// rows (Solver_CPU_RB.cpp:155-162), and its last CTA to finish runs the
// convergence poll, so one iteration is two launches and no host round trip.
#pragma once
#include <type_traits>

#include "qesb_device.cuh"

namespace qesb {

struct SplitGeom {
  int PQ;    // padded half-row length
  long CS;   // elements per colour array
  __host__ __device__ long row(int j, int k, int Y) const { return ((long)k * Y + j) * PQ; }
};

struct SplitArgs {
  DevGrid G;
  SplitGeom S;
  float *lam;           // [2][CS]
  const float *R;       // [2][CS]
  const uint8_t *mask;  // [2][CS]
  const float *val;     // [6][Z]
  const float *inv;     // [Z][64]
  double *err;
  SolveState *st;
  int itermax;
  double tol;
};

// Convergence poll for the iteration st->it (see k_poll in qesb_solver.cu for
// the loop condition); run by one thread once every CTA's error is in.
__device__ __forceinline__ void poll_one(SolveState *st, const double *err, double tol, int itermax)
{
  const int it = st->it;
  const double e = err[it];
  st->residual = e;
  st->it = it + 1;
  st->cur = 0;
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

// One colour of the sweep over rows j in [1, Y-2], k in [1, Z-2]. Persistent:
// the grid holds as many CTAs as fit on the GPU at once and each warp sweeps a
// contiguous range of rows, so it pays the start-up latency and its share of
// the block reduction once, reloads the per-layer tables only when k changes,
// and never waits on another warp inside the sweep.
template <int COLOUR, int RPB, int U, int STRIDED>
__global__ void __launch_bounds__(32 * RPB) k_sor_split(SplitArgs a)
{
  SolveState *S = a.st;
  if (S->done) return;
  const DevGrid &G = a.G;
  const int it = S->it;
  const int nrows = (G.Y - 2) * (G.Z - 2);
  const int lane = threadIdx.x;
  const float c1 = 1.0f - kOmega;
  float *L = a.lam;
  double dmax = 0.0;    // warp-wide max |dlambda| so far (all lanes hold it)
  float dmax_f = 0.0f;  // largest float <= dmax
  // Row order: STRIDED = 1 sends the warps through the rows together (warp w
  // takes rows w, w + warps, ...), so the rows in flight form one window and
  // DRAM sees a few long streams; STRIDED = 0 gives each warp a contiguous
  // range (fewer per-layer table reloads, scattered streams).
  const int warps = gridDim.x * RPB, w = blockIdx.x * RPB + threadIdx.y;
  const int r_begin = STRIDED ? w : (int)((long)nrows * w / warps);
  const int r_end = STRIDED ? nrows : (int)((long)nrows * (w + 1) / warps);
  const int r_step = STRIDED ? warps : 1;
  int kcur = -1;
  float ve = 0, vf = 0, vg = 0, vh = 0, vm = 0, vn = 0, inv63 = 0;
  const float *inv = a.inv;
  for (int r = r_begin; r < r_end; r += r_step) {
    const int k = 1 + r / (G.Y - 2), j = 1 + r % (G.Y - 2);
    if (k != kcur) {
      kcur = k;
      ve = __ldg(a.val + 0 * G.Z + k);
      vf = __ldg(a.val + 1 * G.Z + k);
      vg = __ldg(a.val + 2 * G.Z + k);
      vh = __ldg(a.val + 3 * G.Z + k);
      vm = __ldg(a.val + 4 * G.Z + k);
      vn = __ldg(a.val + 5 * G.Z + k);
      inv = a.inv + k * 64;
      inv63 = __ldg(inv + 63);
    }
    const int i0 = (COLOUR + j + k) & 1;
    const long own = COLOUR * a.S.CS + a.S.row(j, k, G.Y);
    const long oth = (1 - COLOUR) * a.S.CS + a.S.row(j, k, G.Y);
    // Updated cells of this row: i in [1, X-2], i = i0 + 2q. Every load goes
    // through the read-only path: a cell's own value is read once, by the lane
    // that then writes it; the other colour, R and the mask are not written
    // during this half-sweep except by the ground-mirror copies below, which a
    // warp makes only after its own reads of those cells.
    const int qlo = i0 ? 0 : 1;
    const int qhi = (G.X - 2 - i0) >> 1;  // inclusive
    float *pw = L + own;
    const float *pxm = L + oth + i0 - 1;
    const float *pxp = L + oth + i0;
    const float *pym = L + oth - a.S.PQ;
    const float *pyp = L + oth + a.S.PQ;
    const float *pzm = L + oth - (long)G.Y * a.S.PQ;
    const float *pzp = L + oth + (long)G.Y * a.S.PQ;
    const float *pr = a.R + own;
    const uint8_t *pm = a.mask + own;
    // One batch: U cells per lane at q0b + 32u. PRED: a slot is live only if
    // inside the row (the row's last, partial batch); dead slots load nothing.
    // All-fluid warps skip the wall-mask selects. The error is FP64-exact
    // without converting every cell: rounding is monotone, so
    // fl(|nv - old|) < rd(dmax) proves |nv - old| < dmax; only when some lane
    // fails that test (or holds a NaN) does the warp take the FP64 path.
    auto batch = [&](int q0b, auto pred_tag) {
      constexpr bool PRED = decltype(pred_tag)::value;
      float old[U], xm[U], xp[U], ym[U], yp[U], zm[U], zp[U], rr[U], nv[U];
      unsigned mk[U];
      bool live[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int q = q0b + 32 * u;
        live[u] = !PRED || q <= qhi;
        old[u] = xm[u] = xp[u] = ym[u] = yp[u] = zm[u] = zp[u] = rr[u] = 0.0f;
        mk[u] = 63u;
        if (live[u]) {
          old[u] = __ldg(pw + q);
          xm[u] = __ldg(pxm + q);
          xp[u] = __ldg(pxp + q);
          ym[u] = __ldg(pym + q);
          yp[u] = __ldg(pyp + q);
          zm[u] = __ldg(pzm + q);
          zp[u] = __ldg(pzp + q);
          rr[u] = __ldg(pr + q);
          mk[u] = __ldg(pm + q);
        }
      }
      bool full = true;
#pragma unroll
      for (int u = 0; u < U; ++u) full &= (mk[u] == 63u);
      if (__all_sync(0xffffffffu, full)) {
#pragma unroll
        for (int u = 0; u < U; ++u)
          nv[u] = inv63 * (ve * xp[u] + vf * xm[u] + vg * yp[u] + vh * ym[u] + vm * zp[u] + vn * zm[u] - rr[u]) +
                  c1 * old[u];
      } else {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const unsigned m_ = mk[u];
          const float e = (m_ & 1u) ? ve : 0.0f, f = (m_ & 2u) ? vf : 0.0f;
          const float g = (m_ & 4u) ? vg : 0.0f, hh = (m_ & 8u) ? vh : 0.0f;
          const float m = (m_ & 16u) ? vm : 0.0f, n = (m_ & 32u) ? vn : 0.0f;
          nv[u] = __ldg(inv + m_) * (e * xp[u] + f * xm[u] + g * yp[u] + hh * ym[u] + m * zp[u] + n * zm[u] - rr[u]) +
                  c1 * old[u];
        }
      }
      bool big = false;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (live[u]) {
          pw[q0b + 32 * u] = nv[u];
          big |= !(fabsf(nv[u] - old[u]) < dmax_f);
        }
      }
      if (__any_sync(0xffffffffu, big)) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const double d = fabs((double)nv[u] - (double)old[u]);
          if (live[u] && (d > dmax || d != d)) dmax = d;
        }
        dmax = warp_max_d(dmax);
        dmax_f = __double2float_rd(dmax);
      }
    };
    int q0 = qlo + lane;
    // full batches while every lane's U cells lie inside the row (warp-uniform
    // test on the warp's last lane), then one predicated batch for the rest
    const int lane_off = 31 - lane;
    for (; q0 + lane_off + 32 * (U - 1) <= qhi; q0 += 32 * U) batch(q0, std::false_type{});
    if (q0 - lane <= qhi) batch(q0, std::true_type{});
    if (COLOUR == 1 && k == 1) {
      __syncwarp();  // one warp owns the row: its black updates land before the copies
      // ground mirror of this row, both colours: (i, j, 0) <- (i, j, 1); the
      // plane-0 cell of colour c mirrors the plane-1 cell of colour 1-c at
      // the same q. The black plane-1 values are this warp's own; the red
      // plane-1 values are read-only during this kernel.
      const long b1 = 1 * a.S.CS + a.S.row(j, 1, G.Y), r0 = 0 * a.S.CS + a.S.row(j, 0, G.Y);
      const long r1 = 0 * a.S.CS + a.S.row(j, 1, G.Y), b0 = 1 * a.S.CS + a.S.row(j, 0, G.Y);
      const int qn = (G.X + 1) >> 1;
      for (int q = lane; q < qn; q += 32) {
        L[r0 + q] = L[b1 + q];
        L[b0 + q] = L[r1 + q];
      }
    }
  }
  // block max -> err[it], then (black) last-CTA poll
  __shared__ double s_part[RPB];
  __shared__ bool s_last;
  double v = warp_max_d(dmax);
  if (lane == 0) s_part[threadIdx.y] = v;
  __syncthreads();
  if (threadIdx.y == 0) {
    double x = lane < RPB ? s_part[lane] : 0.0;
    x = warp_max_d(x);
    if (lane == 0) {
      if (x != 0.0) atomic_max_nonneg(a.err + it, x);
      if (COLOUR == 1) {
        __threadfence();
        const unsigned t = atomicAdd(&S->blocks_done, 1u);
        s_last = (t == gridDim.x - 1);
      }
    }
  }
  if (COLOUR == 1) {
    __syncthreads();
    if (s_last && lane == 0 && threadIdx.y == 0) {
      __threadfence();
      S->blocks_done = 0;
      poll_one(S, a.err, a.tol, a.itermax);
    }
  }
}

// Vectorised variant of k_sor_split: each lane updates four consecutive
// same-colour cells q..q+3 (q = 4g) with 16-byte loads and one 16-byte store,
// so a warp moves 512 B per request instead of 128 B. Rows start on 128-byte
// boundaries (PQ is a multiple of 32), so every float4 is aligned. The four
// x-neighbour pairs come from the other colour's float4 at q plus one value
// across the group edge (q-1 when i0 = 0, q+4 when i0 = 1), taken from the
// neighbouring lane by a shuffle, or loaded at the warp's edge. Cells of the
// group outside [qlo, qhi] are rewritten with the value this lane read.
template <int COLOUR, int RPB, int STRIDED>
__global__ void __launch_bounds__(32 * RPB) k_sor_split4(SplitArgs a)
{
  SolveState *S = a.st;
  if (S->done) return;
  const DevGrid &G = a.G;
  const int it = S->it;
  const int nrows = (G.Y - 2) * (G.Z - 2);
  const int lane = threadIdx.x;
  const float c1 = 1.0f - kOmega;
  float *L = a.lam;
  double dmax = 0.0;
  float dmax_f = 0.0f;
  // Row order: STRIDED = 1 sends the warps through the rows together (warp w
  // takes rows w, w + warps, ...), so the rows in flight form one window and
  // DRAM sees a few long streams; STRIDED = 0 gives each warp a contiguous
  // range (fewer per-layer table reloads, scattered streams).
  const int warps = gridDim.x * RPB, w = blockIdx.x * RPB + threadIdx.y;
  const int r_begin = STRIDED ? w : (int)((long)nrows * w / warps);
  const int r_end = STRIDED ? nrows : (int)((long)nrows * (w + 1) / warps);
  const int r_step = STRIDED ? warps : 1;
  int kcur = -1;
  float ve = 0, vf = 0, vg = 0, vh = 0, vm = 0, vn = 0, inv63 = 0;
  const float *inv = a.inv;
  for (int r = r_begin; r < r_end; r += r_step) {
    const int k = 1 + r / (G.Y - 2), j = 1 + r % (G.Y - 2);
    if (k != kcur) {
      kcur = k;
      ve = __ldg(a.val + 0 * G.Z + k);
      vf = __ldg(a.val + 1 * G.Z + k);
      vg = __ldg(a.val + 2 * G.Z + k);
      vh = __ldg(a.val + 3 * G.Z + k);
      vm = __ldg(a.val + 4 * G.Z + k);
      vn = __ldg(a.val + 5 * G.Z + k);
      inv = a.inv + k * 64;
      inv63 = __ldg(inv + 63);
    }
    const int i0 = (COLOUR + j + k) & 1;
    const long own = COLOUR * a.S.CS + a.S.row(j, k, G.Y);
    const long oth = (1 - COLOUR) * a.S.CS + a.S.row(j, k, G.Y);
    const int qlo = i0 ? 0 : 1;
    const int qhi = (G.X - 2 - i0) >> 1;  // inclusive
    float *pw = L + own;
    const float *px = L + oth;
    const float *pym = L + oth - a.S.PQ;
    const float *pyp = L + oth + a.S.PQ;
    const float *pzm = L + oth - (long)G.Y * a.S.PQ;
    const float *pzp = L + oth + (long)G.Y * a.S.PQ;
    const float *pr = a.R + own;
    const uint8_t *pm = a.mask + own;
    // warp-uniform loop over 128-cell spans; lane g-th group is live if its
    // first cell is inside the row (live lanes form a prefix of the warp)
    for (int g0 = 0; 4 * g0 <= qhi; g0 += 32) {
      const int q = 4 * (g0 + lane);
      const bool live = q <= qhi;
      float4 o = make_float4(0, 0, 0, 0), rr = o, ym = o, yp = o, zm = o, zp = o, xc = o;
      uint32_t m4 = 0x3f3f3f3fu;
      if (live) {
        o = __ldg(reinterpret_cast<const float4 *>(pw + q));
        xc = __ldg(reinterpret_cast<const float4 *>(px + q));
        ym = __ldg(reinterpret_cast<const float4 *>(pym + q));
        yp = __ldg(reinterpret_cast<const float4 *>(pyp + q));
        zm = __ldg(reinterpret_cast<const float4 *>(pzm + q));
        zp = __ldg(reinterpret_cast<const float4 *>(pzp + q));
        rr = __ldg(reinterpret_cast<const float4 *>(pr + q));
        m4 = __ldg(reinterpret_cast<const uint32_t *>(pm + q));
      }
      // value across the group edge: other[q-1] (i0 = 0) or other[q+4] (i0 = 1)
      float edge = i0 ? __shfl_down_sync(0xffffffffu, xc.x, 1) : __shfl_up_sync(0xffffffffu, xc.w, 1);
      if (live) {
        if (i0) {
          if ((lane == 31 || q + 4 > qhi) && q + 3 <= qhi) edge = __ldg(px + q + 4);
        } else {
          if (lane == 0 && q > 0) edge = __ldg(px + q - 1);
        }
      }
      const float xm0 = i0 ? xc.x : edge, xm1 = i0 ? xc.y : xc.x, xm2 = i0 ? xc.z : xc.y, xm3 = i0 ? xc.w : xc.z;
      const float xp0 = i0 ? xc.y : xc.x, xp1 = i0 ? xc.z : xc.y, xp2 = i0 ? xc.w : xc.z, xp3 = i0 ? edge : xc.w;
      // cells of the group that are updated: q + t in [qlo, qhi]
      bool up[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) up[t] = live && q + t >= qlo && q + t <= qhi;
      unsigned mk[4] = {m4 & 0xffu, (m4 >> 8) & 0xffu, (m4 >> 16) & 0xffu, m4 >> 24};
      bool full = true;
#pragma unroll
      for (int t = 0; t < 4; ++t) full &= (!up[t] || mk[t] == 63u);
      const float ov[4] = {o.x, o.y, o.z, o.w};
      const float xmv[4] = {xm0, xm1, xm2, xm3}, xpv[4] = {xp0, xp1, xp2, xp3};
      const float ymv[4] = {ym.x, ym.y, ym.z, ym.w}, ypv[4] = {yp.x, yp.y, yp.z, yp.w};
      const float zmv[4] = {zm.x, zm.y, zm.z, zm.w}, zpv[4] = {zp.x, zp.y, zp.z, zp.w};
      const float rv[4] = {rr.x, rr.y, rr.z, rr.w};
      float nv[4];
      if (__all_sync(0xffffffffu, full)) {
#pragma unroll
        for (int t = 0; t < 4; ++t)
          nv[t] = inv63 * (ve * xpv[t] + vf * xmv[t] + vg * ypv[t] + vh * ymv[t] + vm * zpv[t] + vn * zmv[t] - rv[t]) +
                  c1 * ov[t];
      } else {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const unsigned m_ = up[t] ? mk[t] : 63u;
          const float e = (m_ & 1u) ? ve : 0.0f, f = (m_ & 2u) ? vf : 0.0f;
          const float g = (m_ & 4u) ? vg : 0.0f, hh = (m_ & 8u) ? vh : 0.0f;
          const float m = (m_ & 16u) ? vm : 0.0f, n = (m_ & 32u) ? vn : 0.0f;
          nv[t] = __ldg(inv + m_) * (e * xpv[t] + f * xmv[t] + g * ypv[t] + hh * ymv[t] + m * zpv[t] + n * zmv[t] - rv[t]) +
                  c1 * ov[t];
        }
      }
      bool big = false;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        nv[t] = up[t] ? nv[t] : ov[t];
        big |= up[t] && !(fabsf(nv[t] - ov[t]) < dmax_f);
      }
      if (live) *reinterpret_cast<float4 *>(pw + q) = make_float4(nv[0], nv[1], nv[2], nv[3]);
      if (__any_sync(0xffffffffu, big)) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const double d = fabs((double)nv[t] - (double)ov[t]);
          if (up[t] && (d > dmax || d != d)) dmax = d;
        }
        dmax = warp_max_d(dmax);
        dmax_f = __double2float_rd(dmax);
      }
    }
    if (COLOUR == 1 && k == 1) {
      __syncwarp();  // one warp owns the row: its black updates land before the copies
      const long b1 = 1 * a.S.CS + a.S.row(j, 1, G.Y), r0 = 0 * a.S.CS + a.S.row(j, 0, G.Y);
      const long r1 = 0 * a.S.CS + a.S.row(j, 1, G.Y), b0 = 1 * a.S.CS + a.S.row(j, 0, G.Y);
      const int qn = (G.X + 1) >> 1;
      for (int qq = lane; qq < qn; qq += 32) {
        L[r0 + qq] = L[b1 + qq];
        L[b0 + qq] = L[r1 + qq];
      }
    }
  }
  __shared__ double s_part[RPB];
  __shared__ bool s_last;
  double v = warp_max_d(dmax);
  if (lane == 0) s_part[threadIdx.y] = v;
  __syncthreads();
  if (threadIdx.y == 0) {
    double x = lane < RPB ? s_part[lane] : 0.0;
    x = warp_max_d(x);
    if (lane == 0) {
      if (x != 0.0) atomic_max_nonneg(a.err + it, x);
      if (COLOUR == 1) {
        __threadfence();
        const unsigned t = atomicAdd(&S->blocks_done, 1u);
        s_last = (t == gridDim.x - 1);
      }
    }
  }
  if (COLOUR == 1) {
    __syncthreads();
    if (s_last && lane == 0 && threadIdx.y == 0) {
      __threadfence();
      S->blocks_done = 0;
      poll_one(S, a.err, a.tol, a.itermax);
    }
  }
}

// Plane-0 boundary ring (j = 0, Y-1 rows; i = 0, X-1 columns) <- plane 1.
// Those plane-0 cells are read by no update (their plane-1 partners are
// boundary cells, never updated, whose values never change), so mirroring them
// once after the iterations leaves the same field as mirroring every iteration.
__global__ void k_split_mirror_ring(DevGrid G, SplitGeom S, float *lam)
{
  const int j = blockIdx.x;
  const bool edge_row = (j == 0 || j == G.Y - 1);
  const int qn = (G.X + 1) >> 1;
  for (int c = 0; c < 2; ++c) {
    const long dst = c * S.CS + S.row(j, 0, G.Y), src = (1 - c) * S.CS + S.row(j, 1, G.Y);
    for (int q = threadIdx.x; q < qn; q += blockDim.x) {
      // x of this plane-0 cell: row (j, 0) of colour c has i0 = (c + j) & 1
      const int i = 2 * q + ((c + j) & 1);
      if (i >= G.X) continue;
      if (edge_row || i == 0 || i == G.X - 1) lam[dst + q] = lam[src + q];
    }
  }
}

// Padded natural layout <-> split layout (one thread per cell).
__global__ void k_pad_to_split(DevGrid G, SplitGeom S, const float *__restrict__ src, float *__restrict__ dst)
{
  const int j = blockIdx.y, k = blockIdx.z;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x)
    dst[((i + j + k) & 1) * S.CS + S.row(j, k, G.Y) + (i >> 1)] = src[G.pad(i, j, k)];
}
__global__ void k_split_to_pad(DevGrid G, SplitGeom S, const float *__restrict__ src, float *__restrict__ dst)
{
  const int j = blockIdx.y, k = blockIdx.z;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x)
    dst[G.pad(i, j, k)] = src[((i + j + k) & 1) * S.CS + S.row(j, k, G.Y) + (i >> 1)];
}
__global__ void k_pad_to_split_u8(DevGrid G, SplitGeom S, const uint8_t *__restrict__ src, uint8_t *__restrict__ dst)
{
  const int j = blockIdx.y, k = blockIdx.z;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x)
    dst[((i + j + k) & 1) * S.CS + S.row(j, k, G.Y) + (i >> 1)] = src[G.pad(i, j, k)];
}

}  // namespace qesb
