// Red/black half-sweeps that march in z over tiles of the split layout, with
// the other colour staged once through shared memory (a 2.5D stencil).
//
// A work unit (tile) is 128 cells of a colour row (q in [q0, q0 + 128)),
// TY rows (j in [j0, j0 + TY)) and kc planes (k in [k0, k0 + kc)) of one
// domain. The CTA has TY warps; warp w updates row j0 + w, lane l the cells
// q0 + 4l .. q0 + 4l + 3, one plane after the other. Per plane the CTA stages,
// with 16-byte cp.async copies (zero-filled outside the arrays' rows):
//   - the other colour's plane k + 1 over rows j0 - 1 .. j0 + TY and
//     q0 - 4 .. q0 + 131 (the y and x halos), into a ring of five planes, so
//     planes k - 1, k, k + 1 are resident when plane k is updated;
//   - the own colour's lambda, R and wall mask of plane k, into a ring of three.
// Copies run DIST (1 or 2) planes ahead of the update. Every neighbour then comes from
// shared memory: each byte of the other colour leaves L2 about once per tile
// (plus the halos), against five times in the row kernels.
//
// TMA = 1 stages the same data with tensor-map bulk copies instead: one
// thread per CTA issues, per plane, the other colour's slab (a box of
// 136 x (rows + 2) floats at (q0 - 4, j0 - 1)), the own colour's lambda, R
// and mask rows (boxes of 128 x rows) and the plane's inv row (a 256-byte
// bulk copy), completing on one mbarrier per ring slot; out-of-range box
// elements arrive as zeros, as the zero-filled cp.async copies leave them.
// DIST planes ahead (one or two), the own slots each with their mbarrier.
// The waits are bounded (SweepArgs::wait_limit): a CTA that gives up lets its
// copies in flight land, sets the list's fault flag and stops.
//
// The arithmetic is the row kernels' (Solver_CPU_RB.cpp:118-125, with the
// same operation order), so the results are bit-identical; the black kernel
// applies the ground mirror (Solver_CPU_RB.cpp:155-162) on plane 1 and its
// last CTA runs the convergence poll (qesb_sweep.cuh).
#pragma once
#include <type_traits>

#include "qesb_device.cuh"
#include "qesb_sor_split.cuh"
#include "qesb_sweep.cuh"
#include "qesb_umma.cuh"

namespace qesb {

constexpr int kZmQ = 128;            // colour cells per tile row
constexpr float kZmTinyF = 1.40129846e-45f;  // the smallest positive (subnormal) float
constexpr int kZmOW = kZmQ + 8;      // staged other-colour row: q0 - 4 .. q0 + 131
// Copies run DIST planes ahead of the update (1 or 2): the other colour's ring
// holds planes k - 1 .. k + DIST + 1, the own colour's planes k .. k + DIST.
__host__ __device__ constexpr int zm_other_slots(int dist) { return dist + 3; }
__host__ __device__ constexpr int zm_own_slots(int dist) { return dist + 1; }

// Floats per other-colour slot: the staged slab, rounded up to 128 bytes for
// the TMA shapes (a tensor copy's shared-memory destination is 128-byte aligned).
template <int TR, int TMA>
__host__ __device__ constexpr int zm_oslot_floats()
{
  return TMA ? ((TR + 2) * kZmOW * 4 + 127) / 128 * 32 : (TR + 2) * kZmOW;
}

template <int TR, int DIST, int TMA = 0>
constexpr size_t zm_smem_bytes()
{
  return sizeof(float) * zm_other_slots(DIST) * zm_oslot_floats<TR, TMA>() +
         zm_own_slots(DIST) * TR * kZmQ * (2 * sizeof(float) + 1) + sizeof(float) * zm_own_slots(DIST) * 64 +
         (TMA ? 8 * zm_own_slots(DIST) : 0);
}

__host__ __device__ constexpr int zm_wrap_n(int x, int n) { return x >= n ? x - n : x; }

// 16-byte asynchronous copy global -> shared; src_bytes = 0 fills zeros and
// reads nothing.
__device__ __forceinline__ void zm_cp16(void *dst, const void *src, int src_bytes)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(umma::smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void zm_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void zm_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void zm_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <int TY>
struct ZmSmem {
  float *oth;     // [other slots][ostride]: TY + 2 rows of kZmOW
  float *own;     // [own slots][TY][kZmQ]
  float *rr;      // [own slots][TY][kZmQ]
  uint8_t *mask;  // [own slots][TY][kZmQ]
  float *inv;     // [own slots][64]: omega / (sum of the open faces' coefficients) per wall mask
  uint64_t *bar;  // TMA shapes: [own slots] mbarriers, one per pipeline step in flight
  __device__ ZmSmem(unsigned char *base, int nso, int nsw, int ostride)
  {
    oth = reinterpret_cast<float *>(base);
    own = oth + nso * ostride;
    rr = own + nsw * TY * kZmQ;
    mask = reinterpret_cast<uint8_t *>(rr + nsw * TY * kZmQ);
    inv = reinterpret_cast<float *>(mask + nsw * TY * kZmQ);
    bar = reinterpret_cast<uint64_t *>(inv + nsw * 64);
  }
};

// 4-D tiled tensor copy global -> shared, completing on an mbarrier (no
// multicast: this GPU's own memory only).
__device__ __forceinline__ void zm_tma4(void *dst, const TmaDesc *map, int c0, int c1, int c2, int c3,
                                        uint64_t *mbar)
{
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(umma::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(umma::smem_u32(mbar))
      : "memory");
}
__device__ __forceinline__ void zm_expect_tx(uint64_t *mbar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(umma::smem_u32(mbar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void zm_bulk(void *dst, const void *src, uint32_t bytes, uint64_t *mbar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   umma::smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(umma::smem_u32(mbar))
               : "memory");
}

// The TMA shapes' pipeline step for plane p of a tile (one thread): the own
// colour's lambda, R and mask rows of plane p into own slot `wslot`, the
// other colour's slab of plane p + 1 into other slot `oslot` and, for the
// tile's first plane (first = true), also planes p - 1 and p into the two
// slots before it; the plane's inv row. All on the mbarrier `bar`.
template <int COLOUR, int TR, int OSTR, int NSO>
__device__ __forceinline__ void zm_tma_step(const ZmSmem<TR> &sm, const SplitDom &D, int q0, int j0, int p,
                                            bool first, int oslot, int wslot, uint64_t *bar)
{
  constexpr uint32_t ob = (TR + 2) * kZmOW * 4, wb = TR * kZmQ * 4;
  umma::fence_smem_async();  // the slots' last readers (generic proxy) are done: the barrier before this
  zm_expect_tx(bar, ob * (first ? 3u : 1u) + 2u * wb + TR * kZmQ + 256u);
  const int oc = 1 - COLOUR;
  if (first) {
    zm_tma4(sm.oth + zm_wrap_n(oslot + NSO - 2, NSO) * OSTR, D.tm + kTmOther, q0 - 4, j0 - 1, p - 1, oc, bar);
    zm_tma4(sm.oth + zm_wrap_n(oslot + NSO - 1, NSO) * OSTR, D.tm + kTmOther, q0 - 4, j0 - 1, p, oc, bar);
  }
  zm_tma4(sm.oth + oslot * OSTR, D.tm + kTmOther, q0 - 4, j0 - 1, p + 1, oc, bar);
  zm_tma4(sm.own + wslot * TR * kZmQ, D.tm + kTmOwn, q0, j0, p, COLOUR, bar);
  zm_tma4(sm.rr + wslot * TR * kZmQ, D.tm + kTmR, q0, j0, p, COLOUR, bar);
  zm_tma4(sm.mask + wslot * TR * kZmQ, D.tm + kTmMask, q0, j0, p, COLOUR, bar);
  zm_bulk(sm.inv + wslot * 64, D.inv_all + (long)p * 64, 256u, bar);
}

// A thread's share of a tile's staging, fixed for the tile: shared-memory
// offsets within a slot and global offsets within a colour plane (valid ones
// only; the others zero-fill). Each plane then costs a few adds per copy.
// TR: rows per tile; NT: threads of the CTA.
template <int TR, int NT>
struct ZmCopies {
  static constexpr int NCH = kZmOW / 4;                   // 16-byte chunks per staged row
  static constexpr int NOTH = (TR + 2) * NCH;             // other-colour chunks per plane
  static constexpr int NO = (NOTH + NT - 1) / NT;         // other-colour chunks per thread
  static constexpr int NL = TR * 32 / NT;                 // own lambda / R chunks per thread
  static constexpr int NM = (TR * 8 + NT - 1) / NT;       // own mask chunks per thread
  static_assert(TR * 32 % NT == 0, "own-colour rows must split evenly over the threads");
  int os[NO], og[NO];  // other colour: slot offset (floats), plane offset (floats; -1: zero-fill)
  int ls[NL], lg[NL];  // own lambda and R
  int ms[NM], mg[NM];  // own mask (ms < 0: none)

  __device__ __forceinline__ void init(const SplitDom &D, int j0, int q0, int tid)
  {
#pragma unroll
    for (int t = 0; t < NO; ++t) {
      const int c = tid + t * NT;
      const int r = c / NCH, col = c - r * NCH;
      const int j = j0 - 1 + r, q = q0 - 4 + 4 * col;
      os[t] = c < NOTH ? r * kZmOW + 4 * col : -1;
      og[t] = (c < NOTH && j < D.Y && q >= 0 && q < D.PQ) ? j * D.PQ + q : -1;
    }
#pragma unroll
    for (int t = 0; t < NL; ++t) {
      const int c = tid + t * NT;
      const int r = c >> 5, col = c & 31;
      const int j = j0 + r, q = q0 + 4 * col;
      ls[t] = r * kZmQ + 4 * col;
      lg[t] = (j <= D.Y - 2 && q < D.PQ) ? j * D.PQ + q : -1;
    }
#pragma unroll
    for (int t = 0; t < NM; ++t) {
      const int c = tid + t * NT;
      const int r = c >> 3, col = c & 7;
      const int j = j0 + r, q = q0 + 16 * col;
      ms[t] = c < TR * 8 ? r * kZmQ + 16 * col : -1;
      mg[t] = (c < TR * 8 && j <= D.Y - 2 && q < D.PQ) ? j * D.PQ + q : -1;
    }
  }
};

// Stage the other colour's plane p into other-colour slot `slot`.
template <int COLOUR, int TR, int NT>
__device__ __forceinline__ void zm_stage_other(const ZmSmem<TR> &sm, const ZmCopies<TR, NT> &cp, const SplitDom &D,
                                               int p, int slot)
{
  float *dst = sm.oth + slot * (TR + 2) * kZmOW;
  const float *src = D.L + (1 - COLOUR) * D.CS + (long)p * D.Y * D.PQ;
#pragma unroll
  for (int t = 0; t < ZmCopies<TR, NT>::NO; ++t)
    if (cp.os[t] >= 0) zm_cp16(dst + cp.os[t], cp.og[t] >= 0 ? src + cp.og[t] : D.L, cp.og[t] >= 0 ? 16 : 0);
}

// Stage the own colour's lambda, R and mask of plane p, and the plane's
// 64-entry inverse-coefficient row, into own slot `slot`.
template <int COLOUR, int TR, int NT>
__device__ __forceinline__ void zm_stage_own(const ZmSmem<TR> &sm, const ZmCopies<TR, NT> &cp, const SplitDom &D,
                                             int p, int slot)
{
  const long base = COLOUR * D.CS + (long)p * D.Y * D.PQ;
#pragma unroll
  for (int t = 0; t < ZmCopies<TR, NT>::NL; ++t) {
    const int n = cp.lg[t] >= 0 ? 16 : 0;
    const long g = base + (cp.lg[t] >= 0 ? cp.lg[t] : 0);
    zm_cp16(sm.own + slot * TR * kZmQ + cp.ls[t], D.L + g, n);
    zm_cp16(sm.rr + slot * TR * kZmQ + cp.ls[t], D.R + g, n);
  }
#pragma unroll
  for (int t = 0; t < ZmCopies<TR, NT>::NM; ++t)
    if (cp.ms[t] >= 0)
      zm_cp16(sm.mask + slot * TR * kZmQ + cp.ms[t], D.mask + base + (cp.mg[t] >= 0 ? cp.mg[t] : 0),
              cp.mg[t] >= 0 ? 16 : 0);
  const int tid = threadIdx.x + 32 * threadIdx.y;
  if (tid < 16) zm_cp16(sm.inv + slot * 64 + 4 * tid, D.inv_all + (long)p * 64 + 4 * tid, 16);
}

// One pipeline step's copies: the other colour's plane p + 1 and the own
// colour's plane p (p < k1), as one copy group (empty past the tile's end).
template <int COLOUR, int TR, int NT>
__device__ __forceinline__ void zm_stage(const ZmSmem<TR> &sm, const ZmCopies<TR, NT> &cp, const SplitDom &D, int p,
                                         int k1, int oslot, int wslot)
{
  if (p < k1) {
    zm_stage_other<COLOUR, TR, NT>(sm, cp, D, p + 1, oslot);
    zm_stage_own<COLOUR, TR, NT>(sm, cp, D, p, wslot);
  }
  zm_commit();
}

template <int N>
__device__ __forceinline__ int zm_wrap(int x) { return x >= N ? x - N : x; }

// TY warps per CTA, RW rows per warp (rows w, w + TY, ...): tiles of TY x RW rows;
// copies DIST planes ahead. BAL = 1: the list's units are single planes of a
// tile column (kc = 1, planes fastest) and each CTA takes an equal share of
// them, walked as runs of consecutive planes, so every CTA does the same
// number of plane steps whatever the list's size (one or two runs each, each
// run paying its own pipeline start).
template <int COLOUR, int TY, int RW, int DIST, bool MULTI, int MINB, int TMA = 0, int BAL = 0>
__global__ void __launch_bounds__(32 * TY, MINB) k_sor_zm(SweepArgs b)
{
  constexpr int TR = TY * RW, NT = 32 * TY, NSO = zm_other_slots(DIST), NSW = zm_own_slots(DIST);
  constexpr int OSTR = zm_oslot_floats<TR, TMA>();
  static_assert(DIST == 1 || DIST == 2, "copies run one or two planes ahead");
  pdl_wait_release();
  const int na = b.ctl->nactive;
  if (na <= 0) return;
  extern __shared__ __align__(128) unsigned char zm_raw[];
  const ZmSmem<TR> sm(zm_raw, NSO, NSW, OSTR);
  const int lane = threadIdx.x, w = threadIdx.y, tid = lane + 32 * w;
  [[maybe_unused]] const uint32_t wlim = b.wait_limit ? b.wait_limit : kStageWaitLimit;
  [[maybe_unused]] unsigned nst = 0, nwt = 0;  // TMA pipeline steps issued / waited by this CTA
  [[maybe_unused]] bool tma_bad = false;       // TMA shapes: slots not 128-byte aligned
  if constexpr (TMA) {
    if (tid == 0) {
#pragma unroll
      for (int s2 = 0; s2 < NSW; ++s2) umma::mbar_init(&sm.bar[s2], 1);
      umma::fence_mbar_init();
    }
    tma_bad = (umma::smem_u32(zm_raw) & 127u) != 0;
    __syncthreads();
  }
  const int total = MULTI ? b.uoff[na] : sweep_units(b.one, kUnitTile);
  SplitDom D;
  int slot = -1, lo = 0, hi = 0;
  const int ub = BAL ? (int)((long)total * blockIdx.x / gridDim.x) : (int)blockIdx.x;
  const int ue = BAL ? (int)((long)total * (blockIdx.x + 1) / gridDim.x) : total;
  int unext = ub;
  for (int u = ub; u < ue; u = unext) {
    if (!MULTI) {
      if (slot < 0) {
        slot = 0;
        hi = total;
        D.load(b.one);
      }
    } else if (slot < 0 || u >= hi) {
      if (slot >= 0) D.flush(lane);
      slot = sweep_slot(b.uoff, na, u);
      lo = b.uoff[slot];
      hi = b.uoff[slot + 1];
      D.load(sweep_dom<MULTI>(b, slot));
    }
    if constexpr (TMA) {
      if (tma_bad || D.tm == nullptr) {  // no tensor maps for this domain: stop with the fault flag set
        if (tid == 0) atomicExch(&b.ctl->fault, 1);
        break;
      }
    }
    const SweepDomain &SD = sweep_dom<MULTI>(b, slot);
    const int njt = (D.Y - 2 + TR - 1) / TR;
    const int nch = SD.nch;
    int qt, jt, k0, k1;
    if constexpr (BAL) {  // planes fastest: a run of this column's planes, to the column's end or the share's
      const int P = D.Z - 2, t = u - lo, kt = t % P, col = t / P;
      qt = col % nch;
      jt = col / nch;
      k0 = 1 + kt;
      k1 = 1 + min(P, kt + (ue - u));
      unext = u + (k1 - k0);
    } else {
      const int kc = SD.kc;
      int t = u - lo;
      qt = t % nch;
      t /= nch;
      jt = t % njt;
      k0 = 1 + (t / njt) * kc;
      k1 = min(k0 + kc, D.Z - 1);
      unext = u + (int)gridDim.x;
    }
    const int q0 = qt * kZmQ, j0 = 1 + jt * TR;
    const int q = q0 + 4 * lane;
    const int qn = (D.X + 1) >> 1;
    ZmCopies<TR, NT> cp;
    if constexpr (!TMA) cp.init(D, j0, q0, tid);
    // the lane's updated cells for rows of each x parity: q + t in [qlo, qhi],
    // qlo = 1 - I0, qhi = (X - 2 - I0) / 2
    unsigned up0 = 0, up1 = 0, upb0 = 0, upb1 = 0;  // bit / byte t: cell q + t
#pragma unroll
    for (int t4 = 0; t4 < 4; ++t4) {
      const bool a0 = q + t4 >= 1 && q + t4 <= (D.X - 2) >> 1, a1 = q + t4 <= (D.X - 3) >> 1;
      up0 |= a0 ? 1u << t4 : 0u;
      up1 |= a1 ? 1u << t4 : 0u;
      upb0 |= a0 ? 0xffu << (8 * t4) : 0u;
      upb1 |= a1 ? 0xffu << (8 * t4) : 0u;
    }
    D.dmax_f = fmaxf(D.dmax_f, kZmTinyF);

    // Ring slots restart with each tile: the other colour's plane k0 - 1 + s
    // sits in slot s mod NSO, the own colour's plane k0 + s in slot s mod NSW.
    // Prologue: other planes k0 - 1, k0 (and k0 + 1 with own k0) as one
    // group, then the steps of planes k0 + 1 .. k0 + DIST - 1.
    if constexpr (TMA) {
      if (tid == 0) zm_tma_step<COLOUR, TR, OSTR, NSO>(sm, D, q0, j0, k0, true, 2, 0, &sm.bar[nst % NSW]);
      ++nst;
      if (DIST == 2 && k0 + 1 < k1) {
        if (tid == 0) zm_tma_step<COLOUR, TR, OSTR, NSO>(sm, D, q0, j0, k0 + 1, false, 3, 1, &sm.bar[nst % NSW]);
        ++nst;
      }
    } else {
      zm_stage_other<COLOUR, TR, NT>(sm, cp, D, k0 - 1, 0);
      zm_stage_other<COLOUR, TR, NT>(sm, cp, D, k0, 1);
#pragma unroll
      for (int d = 0; d < DIST; ++d) zm_stage<COLOUR, TR, NT>(sm, cp, D, k0 + d, k1, 2 + d, d);
    }
    int om1 = 0, wk = 0;  // slots of the other colour's plane k - 1 and the own colour's plane k
    // the plane's six face coefficients, loaded one plane ahead
    float lv[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) lv[f] = __ldg(D.val + f * D.Z + k0);
    for (int k = k0; k < k1; ++k, om1 = zm_wrap<NSO>(om1 + 1), wk = zm_wrap<NSW>(wk + 1)) {
      if constexpr (TMA) {
        // plane k's step has landed (bounded wait), and every warp is done with plane k - 1
        const bool ok = umma::mbar_wait_bounded(&sm.bar[nwt % NSW], (nwt / NSW) & 1u, wlim);
        ++nwt;
        if (__syncthreads_or(!ok)) {
          // let every copy of this CTA still in flight land, then stop
          for (unsigned n = nwt - 1; n < nst; ++n) umma::mbar_wait(&sm.bar[n % NSW], (n / NSW) & 1u, kStageWaitLimit);
          if (tid == 0) atomicExch(&b.ctl->fault, 1);
          goto tiles_done;
        }
        if (k + DIST < k1) {
          if (tid == 0)
            zm_tma_step<COLOUR, TR, OSTR, NSO>(sm, D, q0, j0, k + DIST, false, zm_wrap<NSO>(om1 + DIST + 2),
                                               zm_wrap<NSW>(wk + DIST), &sm.bar[nst % NSW]);
          ++nst;
        }
      } else {
        zm_wait<DIST - 1>();  // this thread's copies of plane k's step have landed
        __syncthreads();      // everyone's; and every warp is done with plane k - 1
        zm_stage<COLOUR, TR, NT>(sm, cp, D, k + DIST, k1, zm_wrap<NSO>(om1 + DIST + 2), zm_wrap<NSW>(wk + DIST));
      }
      D.ve = lv[0];
      D.vf = lv[1];
      D.vg = lv[2];
      D.vh = lv[3];
      D.vm = lv[4];
      D.vn = lv[5];
      const float *sinv = sm.inv + wk * 64;
      D.inv63 = sinv[63];
      if (k + 1 < k1) {
#pragma unroll
        for (int f = 0; f < 6; ++f) lv[f] = __ldg(D.val + f * D.Z + k + 1);
      }
      const float *om = sm.oth + om1 * OSTR;
      const float *ok = sm.oth + zm_wrap<NSO>(om1 + 1) * OSTR;
      const float *op = sm.oth + zm_wrap<NSO>(om1 + 2) * OSTR;
      const int c = 4 + 4 * lane;  // column of q in a staged other-colour row
      // One row: I0 = (COLOUR + j + k) & 1, the x parity of the row's cells
      // (cell q is i = 2q + I0), known at compile time in each branch.
      auto row = [&](const int wr, const int j, auto i0_tag) {
        constexpr int I0 = decltype(i0_tag)::value;
        const unsigned upm = I0 ? up1 : up0;  // which of the lane's 4 cells are updated
        const int so = wk * TR * kZmQ + wr * kZmQ + 4 * lane;
        const float4 o = *reinterpret_cast<const float4 *>(sm.own + so);
        const float4 rr = *reinterpret_cast<const float4 *>(sm.rr + so);
        const uint32_t m4 = *reinterpret_cast<const uint32_t *>(sm.mask + so);
        const float4 xc = *reinterpret_cast<const float4 *>(ok + (wr + 1) * kZmOW + c);
        const float4 ym = *reinterpret_cast<const float4 *>(ok + wr * kZmOW + c);
        const float4 yp = *reinterpret_cast<const float4 *>(ok + (wr + 2) * kZmOW + c);
        const float4 zm = *reinterpret_cast<const float4 *>(om + (wr + 1) * kZmOW + c);
        const float4 zp = *reinterpret_cast<const float4 *>(op + (wr + 1) * kZmOW + c);
        // value across the group edge: other[q - 1] (I0 = 0) or other[q + 4] (I0 = 1)
        const float edge = ok[(wr + 1) * kZmOW + (I0 ? c + 4 : c - 1)];
        const float xmv[4] = {I0 ? xc.x : edge, I0 ? xc.y : xc.x, I0 ? xc.z : xc.y, I0 ? xc.w : xc.z};
        const float xpv[4] = {I0 ? xc.y : xc.x, I0 ? xc.z : xc.y, I0 ? xc.w : xc.z, I0 ? edge : xc.w};
        // 6-bit wall masks (the & keeps every table index inside its 64 entries)
        const unsigned mk[4] = {m4 & 0x3fu, (m4 >> 8) & 0x3fu, (m4 >> 16) & 0x3fu, (m4 >> 24) & 0x3fu};
        // all-fluid: every updated cell has all six faces open (mask byte 63)
        const bool full = ((m4 ^ 0x3f3f3f3fu) & (I0 ? upb1 : upb0)) == 0u;
        const float ov[4] = {o.x, o.y, o.z, o.w};
        const float ymv[4] = {ym.x, ym.y, ym.z, ym.w}, ypv[4] = {yp.x, yp.y, yp.z, yp.w};
        const float zmv[4] = {zm.x, zm.y, zm.z, zm.w}, zpv[4] = {zp.x, zp.y, zp.z, zp.w};
        const float rv[4] = {rr.x, rr.y, rr.z, rr.w};
        float nv[4];
        if (__all_sync(0xffffffffu, full)) {
#pragma unroll
          for (int t4 = 0; t4 < 4; ++t4)
            nv[t4] = D.inv63 * (D.ve * xpv[t4] + D.vf * xmv[t4] + D.vg * ypv[t4] + D.vh * ymv[t4] +
                                D.vm * zpv[t4] + D.vn * zmv[t4] - rv[t4]) +
                     D.c1 * ov[t4];
        } else {
#pragma unroll
          for (int t4 = 0; t4 < 4; ++t4) {
            const unsigned m_ = (upm >> t4) & 1u ? mk[t4] : 63u;
            const float e = (m_ & 1u) ? D.ve : 0.0f, f = (m_ & 2u) ? D.vf : 0.0f;
            const float g = (m_ & 4u) ? D.vg : 0.0f, hh = (m_ & 8u) ? D.vh : 0.0f;
            const float m = (m_ & 16u) ? D.vm : 0.0f, n = (m_ & 32u) ? D.vn : 0.0f;
            nv[t4] = sinv[m_] * (e * xpv[t4] + f * xmv[t4] + g * ypv[t4] + hh * ymv[t4] + m * zpv[t4] +
                                 n * zmv[t4] - rv[t4]) +
                     D.c1 * ov[t4];
          }
        }
        // Cells outside [qlo, qhi] keep their value. The error trigger: a
        // change of at least the warp's max so far (thr >= the smallest
        // subnormal, so unchanged cells, whose difference is exactly 0, never
        // trigger; denormals are not flushed in this file, so any change is
        // at least that).
        bool big = false;
#pragma unroll
        for (int t4 = 0; t4 < 4; ++t4) {
          nv[t4] = (upm >> t4) & 1u ? nv[t4] : ov[t4];
          big |= !(fabsf(nv[t4] - ov[t4]) < D.dmax_f);
        }
        if (upm) {
          float *pw = D.L + COLOUR * D.CS + ((long)k * D.Y + j) * D.PQ + q;
          *reinterpret_cast<float4 *>(pw) = make_float4(nv[0], nv[1], nv[2], nv[3]);
        }
        if (COLOUR == 1 && k == 1) {
          // ground mirror of this lane's cells: red (i, j, 0) <- black (i, j, 1),
          // black (i, j, 0) <- red (i, j, 1), for q < qn
          float *r0 = D.L + (long)j * D.PQ;
          float *b0 = D.L + D.CS + (long)j * D.PQ;
          const float xv[4] = {xc.x, xc.y, xc.z, xc.w};
#pragma unroll
          for (int t4 = 0; t4 < 4; ++t4)
            if (q + t4 < qn) {
              r0[q + t4] = nv[t4];
              b0[q + t4] = xv[t4];
            }
        }
        // the warp's running max |dlambda|, FP64-exact as in the row kernels
        if (__any_sync(0xffffffffu, big)) {
#pragma unroll
          for (int t4 = 0; t4 < 4; ++t4) {
            const double d = fabs((double)nv[t4] - (double)ov[t4]);
            if (d > D.dmax || d != d) D.dmax = d;
          }
          D.dmax = warp_max_d(D.dmax);
          D.dmax_f = fmaxf(__double2float_rd(D.dmax), kZmTinyF);
        }
      };
#pragma unroll
      for (int r = 0; r < RW; ++r) {
        const int wr = w + r * TY, j = j0 + wr;
        if (j > D.Y - 2) continue;  // warp-uniform
        if ((COLOUR + j + k) & 1) row(wr, j, std::integral_constant<int, 1>{});
        else row(wr, j, std::integral_constant<int, 0>{});
      }
    }
    if constexpr (!TMA) zm_wait0();
    __syncthreads();  // the ring is reused by the next tile
  }
tiles_done:
  sweep_flush_end<MULTI>(D.dmax, MULTI ? (D.err ? D.err + D.it : nullptr) : b.one.err + b.one.st->it);
  if (COLOUR == 1) sweep_finish_black<kUnitTile, MULTI>(b, na);
}

}  // namespace qesb
