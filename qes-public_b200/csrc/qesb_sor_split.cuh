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
// The kernels sweep a domain list (qesb_sweep.cuh): one domain for a single
// solve, every unfinished domain of a batch otherwise.
#pragma once
#include <type_traits>

#include "qesb_device.cuh"
#include "qesb_sweep.cuh"

namespace qesb {

struct SplitGeom {
  int PQ;    // padded half-row length
  long CS;   // elements per colour array
  __host__ __device__ long row(int j, int k, int Y) const { return ((long)k * Y + j) * PQ; }
};

// The current domain of a warp walking rows of a domain list: its fields,
// per-layer tables, and the warp's running FP64 max|dlambda| for it.
struct SplitDom {
  int X = 0, Y = 0, Z = 0, PQ = 0;
  long CS = 0;
  float *L = nullptr;
  const float *R = nullptr, *val = nullptr, *inv_all = nullptr;
  const uint8_t *mask = nullptr;
  const TmaDesc *tm = nullptr;
  double *err = nullptr;
  int it = 0;
  int kcur = -1;
  float c1 = 0.0f;
  float ve = 0, vf = 0, vg = 0, vh = 0, vm = 0, vn = 0, inv63 = 0;
  const float *inv = nullptr;
  double dmax = 0.0;    // warp-wide max |dlambda| so far (all lanes hold it)
  float dmax_f = 0.0f;  // largest float <= dmax

  __device__ __forceinline__ void load(const SweepDomain &D)
  {
    X = D.X;
    Y = D.Y;
    Z = D.Z;
    PQ = D.PQ;
    CS = D.CS;
    L = D.lam;
    R = D.R;
    mask = D.mask;
    tm = D.tm;
    val = D.val;
    inv_all = D.inv;
    err = D.err;
    it = D.st->it;
    c1 = D.c1;
    kcur = -1;
  }
  __device__ __forceinline__ void layer(int k)
  {
    if (k == kcur) return;
    kcur = k;
    ve = __ldg(val + 0 * Z + k);
    vf = __ldg(val + 1 * Z + k);
    vg = __ldg(val + 2 * Z + k);
    vh = __ldg(val + 3 * Z + k);
    vm = __ldg(val + 4 * Z + k);
    vn = __ldg(val + 5 * Z + k);
    inv = inv_all + k * 64;
    inv63 = __ldg(inv + 63);
  }
  // Folds the warp's max into err[it]; the read skips the atomic when an
  // equal or larger value is already there (the common case).
  __device__ __forceinline__ void flush(int lane)
  {
    const double v = warp_max_d(dmax);
    if (lane == 0 && err && v != 0.0) {
      const double cur = *reinterpret_cast<volatile double *>(err + it);
      if (!(cur >= v)) atomic_max_nonneg(err + it, v);
    }
    dmax = 0.0;
    dmax_f = 0.0f;
  }
  // err[] is poll-read only after every CTA's flushes (last-CTA protocol).
};

// Hint to the TMA engine: bring `bytes` (a multiple of 16, 16-byte aligned
// address) into L2. No completion to wait for and no shared memory.
__device__ __forceinline__ void l2_prefetch_bulk(const void *p, unsigned bytes)
{
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// L2 prefetch of the streams a half-sweep of colour `colour` first touches on
// row (j, k): its own lambda, R and mask rows, and the other colour's row
// k + 1 (rows k and k - 1 of the other colour were the z+1 neighbours of
// earlier rows in window order). Rows start on 128-byte boundaries (PQ is a
// multiple of 32), so every address and size is a multiple of 16 bytes; k + 1
// is at most Z - 1, inside the colour array.
__device__ __forceinline__ void split_prefetch_row(const SplitDom &D, int colour, int j, int k)
{
  const long own = colour * D.CS + ((long)k * D.Y + j) * D.PQ;
  const long zp = (1 - colour) * D.CS + ((long)(k + 1) * D.Y + j) * D.PQ;
  const unsigned nb = 4u * (unsigned)D.PQ;
  l2_prefetch_bulk(D.L + own, nb);
  l2_prefetch_bulk(D.R + own, nb);
  l2_prefetch_bulk(D.mask + own, (unsigned)D.PQ);
  l2_prefetch_bulk(D.L + zp, nb);
}

// Walks the rows r of the warp's share of the flattened active-row space,
// switching domain (and flushing the error) when r leaves the current one.
// Calls body(D, j, k) for each row. STRIDED = 2 is window order with an L2
// prefetch, before each row, of the warp's next row (one window ahead), so
// each SM keeps far more DRAM bytes in flight than its loads in registers.
template <int RPB, int STRIDED, bool MULTI, class Body>
__device__ __forceinline__ void split_rows(const SweepArgs &b, int na, SplitDom &D, Body body, int colour)
{
  const int lane = threadIdx.x;
  const int nrows = MULTI ? b.uoff[na] : b.one.rows;
  // Row order: STRIDED = 1 sends the warps through the rows together (warp w
  // takes rows w, w + warps, ...), so the rows in flight form one window and
  // DRAM sees a few long streams; STRIDED = 0 gives each warp a contiguous
  // range (fewer per-layer table reloads, scattered streams).
  const int warps = gridDim.x * RPB, w = blockIdx.x * RPB + threadIdx.y;
  const int r_begin = STRIDED ? w : (int)((long)nrows * w / warps);
  const int r_end = STRIDED ? nrows : (int)((long)nrows * (w + 1) / warps);
  const int r_step = STRIDED ? warps : 1;
  if (r_begin >= r_end) return;
  int slot = MULTI ? sweep_slot(b.uoff, na, r_begin) : 0;
  int lo = MULTI ? b.uoff[slot] : 0, hi = MULTI ? b.uoff[slot + 1] : nrows;
  D.load(sweep_dom<MULTI>(b, slot));
  for (int r = r_begin; r < r_end; r += r_step) {
    if (MULTI && r >= hi) {
      D.flush(lane);
      while (r >= hi) {
        ++slot;
        lo = hi;
        hi = b.uoff[slot + 1];
      }
      D.load(sweep_dom<MULTI>(b, slot));
    }
    const int local = r - lo;
    const int k = 1 + local / (D.Y - 2), j = 1 + local % (D.Y - 2);
    if (STRIDED == 2 && lane == 0 && r + r_step < (MULTI ? min(r_end, hi) : r_end)) {
      const int l2 = local + r_step;
      split_prefetch_row(D, colour, 1 + l2 % (D.Y - 2), 1 + l2 / (D.Y - 2));
    }
    D.layer(k);
    body(j, k);
  }
}

// Ground mirror of row j after its black update, both colours:
// (i, j, 0) <- (i, j, 1) (Solver_CPU_RB.cpp:155-162). The plane-0 cell of
// colour c mirrors the plane-1 cell of colour 1-c at the same q. The black
// plane-1 values are this warp's own; the red ones are read-only during the
// black kernel.
__device__ __forceinline__ void split_mirror_row(const SplitDom &D, int j, int lane)
{
  __syncwarp();  // one warp owns the row: its black updates land before the copies
  const long b1 = 1 * D.CS + ((long)1 * D.Y + j) * D.PQ, r0 = 0 * D.CS + (long)j * D.PQ;
  const long r1 = 0 * D.CS + ((long)1 * D.Y + j) * D.PQ, b0 = 1 * D.CS + (long)j * D.PQ;
  const int qn = (D.X + 1) >> 1;
  for (int q = lane; q < qn; q += 32) {
    D.L[r0 + q] = D.L[b1 + q];
    D.L[b0 + q] = D.L[r1 + q];
  }
}

// One colour of the sweep over rows j in [1, Y-2], k in [1, Z-2] of every
// unfinished domain. Persistent: the grid holds as many CTAs as fit on the
// GPU at once and each warp sweeps its share of the rows, so it pays the
// start-up latency once, reloads the per-layer tables only when k changes,
// and never waits on another warp inside the sweep.
template <int COLOUR, int RPB, int U, int STRIDED, bool MULTI, int MINB = (16 / RPB > 1 ? 16 / RPB : 1)>
__global__ void __launch_bounds__(32 * RPB, MINB) k_sor_split(SweepArgs b)
{
  const int na = b.ctl->nactive;
  if (na <= 0) return;
  const int lane = threadIdx.x;
  SplitDom D;
  split_rows<RPB, STRIDED, MULTI>(b, na, D, [&](int j, int k) {
    const int i0 = (COLOUR + j + k) & 1;
    const long own = COLOUR * D.CS + ((long)k * D.Y + j) * D.PQ;
    const long oth = (1 - COLOUR) * D.CS + ((long)k * D.Y + j) * D.PQ;
    // Updated cells of this row: i in [1, X-2], i = i0 + 2q. Every load goes
    // through the read-only path: a cell's own value is read once, by the lane
    // that then writes it; the other colour, R and the mask are not written
    // during this half-sweep except by the ground-mirror copies below, which a
    // warp makes only after its own reads of those cells.
    const int qlo = i0 ? 0 : 1;
    const int qhi = (D.X - 2 - i0) >> 1;  // inclusive
    float *pw = D.L + own;
    const float *pxm = D.L + oth + i0 - 1;
    const float *pxp = D.L + oth + i0;
    const float *pym = D.L + oth - D.PQ;
    const float *pyp = D.L + oth + D.PQ;
    const float *pzm = D.L + oth - (long)D.Y * D.PQ;
    const float *pzp = D.L + oth + (long)D.Y * D.PQ;
    const float *pr = D.R + own;
    const uint8_t *pm = D.mask + own;
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
          mk[u] = __ldg(pm + q) & 63u;  // 6-bit wall mask: table indexes stay inside 64 entries
        }
      }
      bool full = true;
#pragma unroll
      for (int u = 0; u < U; ++u) full &= (mk[u] == 63u);
      if (__all_sync(0xffffffffu, full)) {
#pragma unroll
        for (int u = 0; u < U; ++u)
          nv[u] = D.inv63 * (D.ve * xp[u] + D.vf * xm[u] + D.vg * yp[u] + D.vh * ym[u] + D.vm * zp[u] +
                             D.vn * zm[u] - rr[u]) +
                  D.c1 * old[u];
      } else {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const unsigned m_ = mk[u];
          const float e = (m_ & 1u) ? D.ve : 0.0f, f = (m_ & 2u) ? D.vf : 0.0f;
          const float g = (m_ & 4u) ? D.vg : 0.0f, hh = (m_ & 8u) ? D.vh : 0.0f;
          const float m = (m_ & 16u) ? D.vm : 0.0f, n = (m_ & 32u) ? D.vn : 0.0f;
          nv[u] = __ldg(D.inv + m_) * (e * xp[u] + f * xm[u] + g * yp[u] + hh * ym[u] + m * zp[u] + n * zm[u] -
                                       rr[u]) +
                  D.c1 * old[u];
        }
      }
      bool big = false;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (live[u]) {
          pw[q0b + 32 * u] = nv[u];
          big |= !(fabsf(nv[u] - old[u]) < D.dmax_f) && nv[u] != old[u];
        }
      }
      if (__any_sync(0xffffffffu, big)) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const double d = fabs((double)nv[u] - (double)old[u]);
          if (live[u] && (d > D.dmax || d != d)) D.dmax = d;
        }
        D.dmax = warp_max_d(D.dmax);
        D.dmax_f = __double2float_rd(D.dmax);
      }
    };
    int q0 = qlo + lane;
    // full batches while every lane's U cells lie inside the row (warp-uniform
    // test on the warp's last lane), then one predicated batch for the rest
    const int lane_off = 31 - lane;
    for (; q0 + lane_off + 32 * (U - 1) <= qhi; q0 += 32 * U) batch(q0, std::false_type{});
    if (q0 - lane <= qhi) batch(q0, std::true_type{});
    if (COLOUR == 1 && k == 1) split_mirror_row(D, j, lane);
  }, COLOUR);
  sweep_flush_end<MULTI>(D.dmax, MULTI ? (D.err ? D.err + D.it : nullptr) : b.one.err + b.one.st->it);
  if (COLOUR == 1) sweep_finish_black<kUnitRow, MULTI>(b, na);
}

// Vectorised variant of k_sor_split: each lane updates four consecutive
// same-colour cells q..q+3 (q = 4g) with 16-byte loads and one 16-byte store,
// so a warp moves 512 B per request instead of 128 B. Rows start on 128-byte
// boundaries (PQ is a multiple of 32), so every float4 is aligned. The four
// x-neighbour pairs come from the other colour's float4 at q plus one value
// across the group edge (q-1 when i0 = 0, q+4 when i0 = 1), taken from the
// neighbouring lane by a shuffle, or loaded at the warp's edge. Cells of the
// group outside [qlo, qhi] are rewritten with the value this lane read.
template <int COLOUR, int RPB, int STRIDED, bool MULTI, int MINB = (16 / RPB > 1 ? 16 / RPB : 1)>
__global__ void __launch_bounds__(32 * RPB, MINB) k_sor_split4(SweepArgs b)
{
  const int na = b.ctl->nactive;
  if (na <= 0) return;
  const int lane = threadIdx.x;
  SplitDom D;
  split_rows<RPB, STRIDED, MULTI>(b, na, D, [&](int j, int k) {
    const int i0 = (COLOUR + j + k) & 1;
    const long own = COLOUR * D.CS + ((long)k * D.Y + j) * D.PQ;
    const long oth = (1 - COLOUR) * D.CS + ((long)k * D.Y + j) * D.PQ;
    const int qlo = i0 ? 0 : 1;
    const int qhi = (D.X - 2 - i0) >> 1;  // inclusive
    float *pw = D.L + own;
    const float *px = D.L + oth;
    const float *pym = D.L + oth - D.PQ;
    const float *pyp = D.L + oth + D.PQ;
    const float *pzm = D.L + oth - (long)D.Y * D.PQ;
    const float *pzp = D.L + oth + (long)D.Y * D.PQ;
    const float *pr = D.R + own;
    const uint8_t *pm = D.mask + own;
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
      unsigned mk[4] = {m4 & 0x3fu, (m4 >> 8) & 0x3fu, (m4 >> 16) & 0x3fu, (m4 >> 24) & 0x3fu};
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
          nv[t] = D.inv63 * (D.ve * xpv[t] + D.vf * xmv[t] + D.vg * ypv[t] + D.vh * ymv[t] + D.vm * zpv[t] +
                             D.vn * zmv[t] - rv[t]) +
                  D.c1 * ov[t];
      } else {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const unsigned m_ = up[t] ? mk[t] : 63u;
          const float e = (m_ & 1u) ? D.ve : 0.0f, f = (m_ & 2u) ? D.vf : 0.0f;
          const float g = (m_ & 4u) ? D.vg : 0.0f, hh = (m_ & 8u) ? D.vh : 0.0f;
          const float m = (m_ & 16u) ? D.vm : 0.0f, n = (m_ & 32u) ? D.vn : 0.0f;
          nv[t] = __ldg(D.inv + m_) * (e * xpv[t] + f * xmv[t] + g * ypv[t] + hh * ymv[t] + m * zpv[t] +
                                       n * zmv[t] - rv[t]) +
                  D.c1 * ov[t];
        }
      }
      bool big = false;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        nv[t] = up[t] ? nv[t] : ov[t];
        big |= up[t] && !(fabsf(nv[t] - ov[t]) < D.dmax_f) && nv[t] != ov[t];
      }
      if (live) *reinterpret_cast<float4 *>(pw + q) = make_float4(nv[0], nv[1], nv[2], nv[3]);
      if (__any_sync(0xffffffffu, big)) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const double d = fabs((double)nv[t] - (double)ov[t]);
          if (up[t] && (d > D.dmax || d != d)) D.dmax = d;
        }
        D.dmax = warp_max_d(D.dmax);
        D.dmax_f = __double2float_rd(D.dmax);
      }
    }
    if (COLOUR == 1 && k == 1) split_mirror_row(D, j, lane);
  }, COLOUR);
  sweep_flush_end<MULTI>(D.dmax, MULTI ? (D.err ? D.err + D.it : nullptr) : b.one.err + b.one.st->it);
  if (COLOUR == 1) sweep_finish_black<kUnitRow, MULTI>(b, na);
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
