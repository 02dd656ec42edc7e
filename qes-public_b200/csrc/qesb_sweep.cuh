// Domain lists for the red/black half-sweep kernels: one solve is a list of
// one domain, a batched solve (qesb_solve_batch) a list of many. The sweep
// kernels spread the work units (rows, 128-cell row spans, or z-march tiles)
// of the unfinished domains over a persistent grid; the last CTA of each black
// launch polls every unfinished domain (the loop condition of
// Solver_CPU_RB.cpp:106, with max|dlambda| in FP64) and compacts the list,
// so finished domains drop out of the next launch without a host round trip.
#pragma once
#include "qesb_device.cuh"

namespace qesb {

// A tensor map (CUtensorMap: 128 bytes, 64-byte aligned) as the TMA copies
// read it from global memory.
struct alignas(64) TmaDesc {
  unsigned long long w[16];
};
// A domain's tensor maps for the TMA z-march shapes, over its split arrays
// as 4-D tensors (q, j, k, colour): the other colour's slab (a box of
// 136 x (rows + 2)), the own colour's lambda and R (128 x rows), the mask.
enum { kTmOther = 0, kTmOwn = 1, kTmR = 2, kTmMask = 3, kTmCount = 4, kTmSlots = 4 };

// One domain in the red/black split layout, as the sweep kernels see it.
struct SweepDomain {
  int X, Y, Z, PQ;
  long CS;
  int nch;    // 128-cell spans per colour row: ceil(PQ / 128)
  int rows;   // (Y - 2) * (Z - 2) updated rows per colour
  int tile_y; // z-march tiles: rows per tile (the kernel's warps per CTA)
  int kc;     // z-march tiles: planes per tile
  float *lam;           // [2][CS]
  const float *R;       // [2][CS]
  const uint8_t *mask;  // [2][CS]
  const float *val;     // [6][Z]
  const float *inv;     // [Z][64]
  double *err;          // [itermax] FP64 max|dlambda| per iteration
  SolveState *st;
  int itermax;
  double tol;
  float c1;  // 1 - omega (omega/sum sits in inv): the reference's 1.78f, or a pre-phase's
  // Window rule (off when wK = 0): after every wK-th iteration of the loop the
  // domain stops if the FP64 max|lambda - snap| over its wn floats is <= wtol;
  // snap then takes lambda's values for the next window.
  int wK;
  long wn;
  double wtol;
  float *snap;
  const TmaDesc *tm;  // [kTmCount] device tensor maps (TMA z-march shapes), or null
};

// Programmatic dependent launch: a list kernel launched while the previous
// one still runs waits here until that grid has completed and its memory is
// visible (a no-op for a plain launch), then lets the next kernel's CTAs be
// scheduled as its own CTAs finish. Every list kernel reads the control block
// and lambda the previous one wrote, so this is its first statement.
__device__ __forceinline__ void pdl_wait_release()
{
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

struct SweepCtl {
  unsigned blocks_done;   // CTAs of the current black launch that have finished
  int nactive;            // domains still iterating
  int fault;              // a bounded stage wait gave up (the launch's results are void)
  int pad;
  unsigned long long t0;  // %globaltimer at the start of the batch
};

// Polls of an mbarrier before a staged kernel's stage wait gives up, sets
// SweepCtl::fault and returns (unless the handle's "wait_limit" option sets
// another count).
constexpr uint32_t kStageWaitLimit = 1u << 22;

struct SweepArgs {
  const SweepDomain *dom;  // [n]
  int *active;             // [n]: indices of the unfinished domains, in batch order
  int *uoff;               // [n + 1]: work-unit offsets over `active`
  SweepCtl *ctl;
  unsigned wait_limit;     // polls before a stage wait gives up (0: kStageWaitLimit)
  SweepDomain one;         // the domain of a single solve, read from the kernel
                           // parameters by the MULTI = false instances
};

// Domain of active slot `slot` (MULTI) or the single solve's domain.
template <bool MULTI>
__device__ __forceinline__ const SweepDomain &sweep_dom(const SweepArgs &b, int slot)
{
  return MULTI ? b.dom[b.active[slot]] : b.one;
}

// Convergence poll for the iteration st->it (Solver_CPU_RB.cpp:106: the loop
// runs while iter < itermax and max_error > tol); one thread per domain.
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

// Kinds of work unit: a row, a 128-cell row span, or a z-march tile
// (128 cells of a colour row x tile_y rows x kc planes).
enum SweepUnit { kUnitRow = 0, kUnitSpan = 1, kUnitTile = 2 };

// Work units of a domain for a kernel family.
__host__ __device__ __forceinline__ int sweep_units(const SweepDomain &D, int unit)
{
  if (unit == kUnitSpan) return D.rows * D.nch;
  if (unit == kUnitTile) return D.nch * ((D.Y - 2 + D.tile_y - 1) / D.tile_y) * ((D.Z - 2 + D.kc - 1) / D.kc);
  return D.rows;
}

// Window rule poll of one domain after a window check gathered its drift:
// the stop when max|lambda - snapshot| <= wtol (converged = 2), NaN as in
// poll_one. One thread per domain.
__device__ __forceinline__ void window_poll_one(const SweepDomain &D)
{
  SolveState *st = D.st;
  const double d = *reinterpret_cast<volatile double *>(&st->wacc);
  st->wacc = 0.0;
  st->wdrift = d;
  if (isnan(d)) {
    st->done = 1;
    st->nan = 1;
  } else if (d <= D.wtol) {
    st->done = 1;
    st->converged = 2;
  }
}

// The last CTA of a launch (blocks counted in ctl->blocks_done, `nblocks` in
// all) polls every active domain with `poll` and rebuilds the active list and
// unit offsets for the next launch. Every thread of the CTA calls it.
template <int UNIT, bool MULTI, typename Poll>
__device__ __forceinline__ void sweep_last_cta_poll(const SweepArgs &b, int na, unsigned nblocks, Poll poll)
{
  __syncthreads();
  const int tid = threadIdx.x + threadIdx.y * blockDim.x, lane = tid & 31;
  if (tid >= 32) return;
  unsigned last = 0;
  if (lane == 0) {
    __threadfence();
    last = atomicAdd(&b.ctl->blocks_done, 1u) == nblocks - 1;
  }
  last = __shfl_sync(0xffffffffu, last, 0);
  if (!last) return;
  __threadfence();
  if (!MULTI) {
    if (lane == 0) {
      if (na > 0) poll(b.one);
      const bool done = na <= 0 || b.one.st->done;
      if (done && na > 0) b.one.st->t_done = global_ns();
      b.ctl->nactive = done ? 0 : 1;
      b.ctl->blocks_done = 0;
    }
    return;
  }
  int out = 0, base = 0;
  for (int a0 = 0; a0 < na; a0 += 32) {
    const int a = a0 + lane;
    int d = -1, keep = 0, units = 0;
    if (a < na) {
      d = b.active[a];
      const SweepDomain &D = b.dom[d];
      poll(D);
      keep = !D.st->done;
      if (!keep) D.st->t_done = global_ns();
      units = sweep_units(D, UNIT);
    }
    __syncwarp();
    const unsigned mball = __ballot_sync(0xffffffffu, keep);
    const int pos = out + __popc(mball & ((1u << lane) - 1u));
    int x = keep ? units : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (keep) {
      b.active[pos] = d;
      b.uoff[pos + 1] = base + x;
    }
    out += __popc(mball);
    base += __shfl_sync(0xffffffffu, x, 31);
  }
  if (lane == 0) {
    b.uoff[0] = 0;
    b.ctl->nactive = out;
    b.ctl->blocks_done = 0;
  }
}

// End of a black launch. Every thread of the CTA calls it after its own error
// flushes; the last CTA to arrive polls the unfinished domains (the loop
// condition) and rebuilds the active list and unit offsets for the next launch.
template <int UNIT, bool MULTI>
__device__ __forceinline__ void sweep_finish_black(const SweepArgs &b, int na)
{
  sweep_last_cta_poll<UNIT, MULTI>(b, na, gridDim.x, [](const SweepDomain &D) {
    poll_one(D.st, D.err, D.tol, D.itermax);
  });
}

// Window check after every wK-th black launch of a loop (every active domain
// then stands at the same iteration, a multiple of wK). blockIdx.y = active
// slot; the CTAs of a slot compare lambda with the domain's snapshot, FP64
// exact, copy lambda into the snapshot and fold the max into st->wacc; the
// last CTA applies the window rule and compacts the list.
template <int UNIT, bool MULTI>
__global__ void __launch_bounds__(256) k_window_check(SweepArgs b)
{
  pdl_wait_release();
  const int na = b.ctl->nactive;
  const int slot = blockIdx.y;
  double dmax = 0.0;
  double *dst = nullptr;
  if (slot < na) {
    const SweepDomain &D = sweep_dom<MULTI>(b, slot);
    if (D.wK > 0) {
      dst = &D.st->wacc;
      const float4 *L = reinterpret_cast<const float4 *>(D.lam);
      float4 *S = reinterpret_cast<float4 *>(D.snap);
      const long n4 = D.wn >> 2;
      for (long i = threadIdx.x + (long)blockIdx.x * blockDim.x; i < n4; i += (long)gridDim.x * blockDim.x) {
        const float4 a = L[i], o = S[i];
        const double d[4] = {fabs((double)a.x - (double)o.x), fabs((double)a.y - (double)o.y),
                             fabs((double)a.z - (double)o.z), fabs((double)a.w - (double)o.w)};
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (d[q] > dmax || d[q] != d[q]) dmax = d[q];
        S[i] = a;
      }
    }
  }
  block_max_to(dst, dmax);
  sweep_last_cta_poll<UNIT, MULTI>(b, na, gridDim.x * gridDim.y, [](const SweepDomain &D) {
    if (D.wK > 0) window_poll_one(D);
  });
}

// Slot of `active` holding unit u: the last slot with uoff[slot] <= u.
__device__ __forceinline__ int sweep_slot(const int *uoff, int na, int u)
{
  int lo = 0, hi = na - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (uoff[mid] <= u) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Last error fold of a launch into dst (the domain's err[it]). A single
// solve's warps all work on one domain: their maxima meet in shared memory
// and the CTA makes one atomic. A list's warps may be on different domains:
// each warp folds its own, skipping the atomic when dst already holds as
// much. Every thread of the CTA calls it; dst may be null for warps of a list
// that had no rows.
template <bool MULTI>
__device__ __forceinline__ void sweep_flush_end(double dmax, double *dst)
{
  const int lane = threadIdx.x & 31;
  const double v = warp_max_d(dmax);
  if (MULTI) {
    if (lane == 0 && dst && v != 0.0) {
      const double cur = *reinterpret_cast<volatile double *>(dst);
      if (!(cur >= v)) atomic_max_nonneg(dst, v);
    }
    return;
  }
  __shared__ double s_part[32];
  const int wid = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
  const int nw = (blockDim.x * blockDim.y) >> 5;
  if (lane == 0) s_part[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double x = lane < nw ? s_part[lane] : 0.0;
    x = warp_max_d(x);
    if (lane == 0 && x != 0.0) atomic_max_nonneg(dst, x);
  }
}

__global__ void k_sweep_stamp(SweepCtl *ctl) { ctl->t0 = global_ns(); }

}  // namespace qesb
