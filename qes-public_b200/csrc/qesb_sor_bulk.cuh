// Bulk-copy staged red/black half-sweeps over a batch of domains (one domain
// for a single solve). Included by qesb_solver.cu, so compiled with
// -fmad=false: each update rounds exactly as Solver_CPU_RB.cpp:118-125 does.
//
// Data: the red/black split layout of qesb_sor_split.cuh (colour arrays of
// 128-byte aligned rows of PQ same-colour cells). Work unit: one 128-cell
// span (chunk c) of one row (j, k) of one domain. Every warp owns a
// contiguous range of units over the batch's unfinished domains and streams
// them through a private ring of NS shared-memory stages: one lane issues the
// unit's bulk copies (cp.async.bulk, global -> shared, completion counted in
// bytes on the stage's mbarrier) NS units ahead of the one being updated, so
// every warp keeps NS units of loads in flight without holding them in
// registers. A stage holds
//     own row span (the cells being updated)            512 B
//     other colour, rows j-1, j, j+1 (+ 4-cell x halo)  <= 1568 B
//     other colour, rows (j, k-1) and (j, k+1)          2 x 512 B
//     R span, wall-mask span                            512 B + 128 B
// When a row is a single chunk (PQ <= 128) rows j-1, j, j+1 are adjacent in
// memory and arrive in one copy. Updated values go straight to global memory
// (16-byte stores); the black kernel also writes the ground mirror
// lambda(k = 0) <- lambda(k = 1) from the values it holds
// (Solver_CPU_RB.cpp:155-162).
//
// Convergence: each warp folds max|dlambda| (FP64-exact, FP32-prefiltered as in
// the split kernels) into its domain's err[it]. The last CTA of the black
// launch polls every unfinished domain (the loop condition of
// Solver_CPU_RB.cpp:106) and compacts the list of unfinished domains and
// their unit offsets, so the next launch spreads only their units over the
// GPU. Finished domains cost nothing; the whole batch needs no host round trip
// until every domain is done.
#pragma once
#include "qesb_device.cuh"
#include "qesb_sweep.cuh"
#include "qesb_umma.cuh"

namespace qesb {

constexpr int kChunk = 128;  // same-colour cells per work unit
// stage layout (bytes)
constexpr int kStOwn = 0;
constexpr int kStOth = 512;                 // 392 floats: 3 x 128 + 8 halo
constexpr int kStZm = kStOth + 392 * 4;     // 2080
constexpr int kStZp = kStZm + 512;          // 2592
constexpr int kStR = kStZp + 512;           // 3104
constexpr int kStMask = kStR + 512;         // 3616
constexpr int kStHdr = kStMask + 128;       // 3744: unit header (domain, j, k, chunk)
constexpr int kStBytes = kStHdr + 16;       // 3760
static_assert(kStBytes % 16 == 0, "stages must keep 16-byte alignment");

using BulkArgs = SweepArgs;

__device__ __forceinline__ void mbar_expect_tx(uint64_t *mbar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(umma::smem_u32(mbar)), "r"(bytes)
               : "memory");
}

// Global -> shared bulk copy (TMA, no tensor map); 16-byte aligned addresses,
// size a multiple of 16; completion adds `bytes` to the mbarrier's tx count.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *mbar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   umma::smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(umma::smem_u32(mbar))
               : "memory");
}

// Per-lane 16-byte asynchronous global -> shared copy (L2 only), grouped per
// unit with commit_group and waited on with wait_group (no spin loop).
__device__ __forceinline__ void lane_g2s16(void *dst, const void *src)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(umma::smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void lane_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void lane_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// The warp copies `bytes` (a multiple of 16) from src to dst, 16 bytes per lane per step.
__device__ __forceinline__ void warp_g2s(unsigned char *dst, const void *src, int bytes, int lane)
{
  const unsigned char *p = static_cast<const unsigned char *>(src);
  for (int o = lane * 16; o < bytes; o += 512) lane_g2s16(dst + o, p + o);
}

template <int W, int NS>
constexpr size_t bulk_smem_bytes()
{
  return (size_t)W * NS * kStBytes + (size_t)W * NS * sizeof(uint64_t);
}

// ASYNC = 0: one lane issues cp.async.bulk copies (TMA engine) completing on
// the stage's mbarrier. ASYNC = 1: every lane issues 16-byte cp.async copies
// (the load/store pipeline), one commit group per unit; the warp waits for
// the oldest group and syncs before reading the stage.
template <int COLOUR, int W, int NS, int ASYNC, bool MULTI>
__global__ void __launch_bounds__(32 * W) k_sor_bulk(BulkArgs b)
{
  extern __shared__ __align__(128) unsigned char smem[];
  const int na = b.ctl->nactive;
  if (na <= 0) return;
  const int lane = threadIdx.x, wid = threadIdx.y;
  const long total = MULTI ? b.uoff[na] : (long)b.one.rows * b.one.nch;
  const long warps = (long)gridDim.x * W, wg = (long)blockIdx.x * W + wid;
  const int ub = (int)(total * wg / warps), ue = (int)(total * (wg + 1) / warps);
  unsigned char *wbase = smem + (size_t)wid * NS * kStBytes;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + (size_t)W * NS * kStBytes) + wid * NS;
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) umma::mbar_init(&bar[s], 1);
    umma::fence_mbar_init();
  }
  __syncwarp();

  // ---- producer cursor (warp-uniform): the next unit to stage -------------
  int pa = MULTI ? sweep_slot(b.uoff, na, ub) : 0;
  int pd = 0, pY = 0, pZ = 0, pPQ = 0, pnch = 1, pj = 1, pk = 1, pc = 0;
  long pCS = 0;
  const float *plam = nullptr, *pR = nullptr;
  const uint8_t *pm = nullptr;
  auto load_dom = [&](int a) {
    pd = MULTI ? b.active[a] : 0;
    const SweepDomain &D = sweep_dom<MULTI>(b, a);
    pY = D.Y;
    pZ = D.Z;
    pPQ = D.PQ;
    pnch = D.nch;
    pCS = D.CS;
    plam = D.lam;
    pR = D.R;
    pm = D.mask;
  };
  if (ub < ue) {
    load_dom(pa);
    const int local = ub - (MULTI ? b.uoff[pa] : 0);
    const int r = local / pnch;
    pc = local - r * pnch;
    pk = 1 + r / (pY - 2);
    pj = 1 + r - (pk - 1) * (pY - 2);
  }
  auto issue = [&](int s) {
    unsigned char *st = wbase + s * kStBytes;
    if (ASYNC) {
      const int q0 = pc * kChunk;
      const int n = min(kChunk, pPQ - q0);
      const long rowo = ((long)pk * pY + pj) * pPQ;
      const float *own = plam + COLOUR * pCS + rowo;
      const float *oth = plam + (1 - COLOUR) * pCS + rowo;
      if (lane == 0) *reinterpret_cast<int4 *>(st + kStHdr) = make_int4(pd, pj, pk, pc);
      const int fb = 4 * n;
      warp_g2s(st + kStOwn, own + q0, fb, lane);
      if (pnch == 1) {
        warp_g2s(st + kStOth, oth - pPQ - 4, 4 * (3 * pPQ + 8), lane);
      } else {
        warp_g2s(st + kStOth, oth + q0 - 4, fb + 32, lane);
        warp_g2s(st + kStOth + 136 * 4, oth - pPQ + q0, fb, lane);
        warp_g2s(st + kStOth + 264 * 4, oth + pPQ + q0, fb, lane);
      }
      warp_g2s(st + kStZm, oth - (long)pY * pPQ + q0, fb, lane);
      warp_g2s(st + kStZp, oth + (long)pY * pPQ + q0, fb, lane);
      warp_g2s(st + kStR, pR + COLOUR * pCS + rowo + q0, fb, lane);
      warp_g2s(st + kStMask, pm + COLOUR * pCS + rowo + q0, n, lane);
    } else if (lane == 0) {
      const int q0 = pc * kChunk;
      const int n = min(kChunk, pPQ - q0);
      const long rowo = ((long)pk * pY + pj) * pPQ;
      const float *own = plam + COLOUR * pCS + rowo;
      const float *oth = plam + (1 - COLOUR) * pCS + rowo;
      *reinterpret_cast<int4 *>(st + kStHdr) = make_int4(pd, pj, pk, pc);
      const uint32_t fb = 4u * n;
      const uint32_t oth_bytes = pnch == 1 ? 4u * (3 * pPQ + 8) : 4u * (3 * n + 8);
      uint64_t *mb = &bar[s];
      mbar_expect_tx(mb, 4 * fb + oth_bytes + (uint32_t)n);
      bulk_g2s(st + kStOwn, own + q0, fb, mb);
      if (pnch == 1) {
        bulk_g2s(st + kStOth, oth - pPQ - 4, 4u * (3 * pPQ + 8), mb);
      } else {
        bulk_g2s(st + kStOth, oth + q0 - 4, fb + 32u, mb);
        bulk_g2s(st + kStOth + 136 * 4, oth - pPQ + q0, fb, mb);
        bulk_g2s(st + kStOth + 264 * 4, oth + pPQ + q0, fb, mb);
      }
      bulk_g2s(st + kStZm, oth - (long)pY * pPQ + q0, fb, mb);
      bulk_g2s(st + kStZp, oth + (long)pY * pPQ + q0, fb, mb);
      bulk_g2s(st + kStR, pR + COLOUR * pCS + rowo + q0, fb, mb);
      bulk_g2s(st + kStMask, pm + COLOUR * pCS + rowo + q0, (uint32_t)n, mb);
    }
    if (ASYNC) lane_commit();
    // advance
    if (++pc == pnch) {
      pc = 0;
      if (++pj == pY - 1) {
        pj = 1;
        if (++pk == pZ - 1) {
          pk = 1;
          if (++pa < na) load_dom(pa);
        }
      }
    }
  };

  // ---- consumer ------------------------------------------------------------
  float c1 = 0.0f;
  int cd = -1, cX = 0, cY = 0, cPQ = 0, cnch = 1, kcur = -1, cit = 0;
  long cCS = 0;
  float *cL = nullptr;
  const float *cval = nullptr, *cinv = nullptr;
  double *cerr = nullptr;
  float ve = 0, vf = 0, vg = 0, vh = 0, vm = 0, vn = 0, inv63 = 0;
  const float *inv = nullptr;
  double dmax = 0.0;
  float dmax_f = 0.0f;
  auto flush = [&]() {
    const double v = warp_max_d(dmax);
    if (lane == 0 && cerr && v != 0.0) {
      const double cur = *reinterpret_cast<volatile double *>(cerr + cit);
      if (!(cur >= v)) atomic_max_nonneg(cerr + cit, v);
    }
    dmax = 0.0;
    dmax_f = 0.0f;
  };

  const int count = ue - ub;
  int issued = 0;
  for (; issued < NS && issued < count; ++issued) issue(issued);
  if (ASYNC)
    for (int e = issued; e < NS; ++e) lane_commit();  // empty groups: one group per slot
  for (int t = 0; t < count; ++t) {
    const int s = t % NS;
    if (ASYNC) {
      lane_wait<NS - 1>();  // this lane's copies of unit t have landed
      __syncwarp();         // and every other lane's
    } else if (!umma::mbar_wait_bounded(&bar[s], (uint32_t)((t / NS) & 1), b.wait_limit ? b.wait_limit : kStageWaitLimit)) {
      if (lane == 0) atomicExch(&b.ctl->fault, 1);
      // let every copy still in flight, this unit's included, land before the
      // CTA's shared memory goes away (bounded by the default limit)
      for (int t2 = t; t2 < issued; ++t2) umma::mbar_wait(&bar[t2 % NS], (uint32_t)((t2 / NS) & 1), kStageWaitLimit);
      break;
    }
    const unsigned char *st = wbase + s * kStBytes;
    const int4 hdr = *reinterpret_cast<const int4 *>(st + kStHdr);
    if (hdr.x != cd) {
      flush();
      cd = hdr.x;
      const SweepDomain &D = MULTI ? b.dom[cd] : b.one;
      cX = D.X;
      cY = D.Y;
      cPQ = D.PQ;
      cnch = D.nch;
      cCS = D.CS;
      cL = D.lam;
      cval = D.val;
      cinv = D.inv;
      cerr = D.err;
      cit = D.st->it;
      c1 = D.c1;
      kcur = -1;
    }
    const int j = hdr.y, k = hdr.z, q0 = hdr.w * kChunk;
    if (k != kcur) {
      kcur = k;
      const int Z = (MULTI ? b.dom[cd] : b.one).Z;
      ve = __ldg(cval + 0 * Z + k);
      vf = __ldg(cval + 1 * Z + k);
      vg = __ldg(cval + 2 * Z + k);
      vh = __ldg(cval + 3 * Z + k);
      vm = __ldg(cval + 4 * Z + k);
      vn = __ldg(cval + 5 * Z + k);
      inv = cinv + k * 64;
      inv63 = __ldg(inv + 63);
    }
    const int i0 = (COLOUR + j + k) & 1;
    const int qlo = i0 ? 0 : 1;
    const int qhi = (cX - 2 - i0) >> 1;  // inclusive
    const int n = min(kChunk, cPQ - q0);
    const float *sown = reinterpret_cast<const float *>(st + kStOwn);
    const float *soth = reinterpret_cast<const float *>(st + kStOth);
    const float *sx, *sym, *syp;
    if (cnch == 1) {
      sym = soth + 4;
      sx = sym + cPQ;
      syp = sx + cPQ;
    } else {
      sx = soth + 4;
      sym = soth + 136;
      syp = soth + 264;
    }
    const int p = 4 * lane;
    const float4 o = *reinterpret_cast<const float4 *>(sown + p);
    const float4 xc = *reinterpret_cast<const float4 *>(sx + p);
    const float4 ym = *reinterpret_cast<const float4 *>(sym + p);
    const float4 yp = *reinterpret_cast<const float4 *>(syp + p);
    const float4 zm = *reinterpret_cast<const float4 *>(reinterpret_cast<const float *>(st + kStZm) + p);
    const float4 zp = *reinterpret_cast<const float4 *>(reinterpret_cast<const float *>(st + kStZp) + p);
    const float4 rr = *reinterpret_cast<const float4 *>(reinterpret_cast<const float *>(st + kStR) + p);
    const uint32_t m4 = reinterpret_cast<const uint32_t *>(st + kStMask)[lane];
    // x neighbour across the 4-cell group edge: other[q - 1] (i0 = 0) or
    // other[q + 4] (i0 = 1); the warp's edge lanes read the stage's halo
    float edge = i0 ? __shfl_down_sync(0xffffffffu, xc.x, 1) : __shfl_up_sync(0xffffffffu, xc.w, 1);
    if (i0 && lane == 31) edge = sx[kChunk];
    if (!i0 && lane == 0) edge = sx[-1];
    const int q = q0 + p;
    const float xm0 = i0 ? xc.x : edge, xm1 = i0 ? xc.y : xc.x, xm2 = i0 ? xc.z : xc.y, xm3 = i0 ? xc.w : xc.z;
    const float xp0 = i0 ? xc.y : xc.x, xp1 = i0 ? xc.z : xc.y, xp2 = i0 ? xc.w : xc.z, xp3 = i0 ? edge : xc.w;
    bool up[4];
#pragma unroll
    for (int t4 = 0; t4 < 4; ++t4) up[t4] = q + t4 >= qlo && q + t4 <= qhi;
    const unsigned mk[4] = {m4 & 0x3fu, (m4 >> 8) & 0x3fu, (m4 >> 16) & 0x3fu, (m4 >> 24) & 0x3fu};
    bool full = true;
#pragma unroll
    for (int t4 = 0; t4 < 4; ++t4) full &= (!up[t4] || mk[t4] == 63u);
    const float ov[4] = {o.x, o.y, o.z, o.w};
    const float xmv[4] = {xm0, xm1, xm2, xm3}, xpv[4] = {xp0, xp1, xp2, xp3};
    const float ymv[4] = {ym.x, ym.y, ym.z, ym.w}, ypv[4] = {yp.x, yp.y, yp.z, yp.w};
    const float zmv[4] = {zm.x, zm.y, zm.z, zm.w}, zpv[4] = {zp.x, zp.y, zp.z, zp.w};
    const float rv[4] = {rr.x, rr.y, rr.z, rr.w};
    float nv[4];
    if (__all_sync(0xffffffffu, full)) {
#pragma unroll
      for (int t4 = 0; t4 < 4; ++t4)
        nv[t4] = inv63 * (ve * xpv[t4] + vf * xmv[t4] + vg * ypv[t4] + vh * ymv[t4] + vm * zpv[t4] + vn * zmv[t4] -
                          rv[t4]) +
                 c1 * ov[t4];
    } else {
#pragma unroll
      for (int t4 = 0; t4 < 4; ++t4) {
        const unsigned m_ = up[t4] ? mk[t4] : 63u;
        const float e = (m_ & 1u) ? ve : 0.0f, f = (m_ & 2u) ? vf : 0.0f;
        const float g = (m_ & 4u) ? vg : 0.0f, hh = (m_ & 8u) ? vh : 0.0f;
        const float m = (m_ & 16u) ? vm : 0.0f, nn = (m_ & 32u) ? vn : 0.0f;
        nv[t4] = __ldg(inv + m_) * (e * xpv[t4] + f * xmv[t4] + g * ypv[t4] + hh * ymv[t4] + m * zpv[t4] +
                                    nn * zmv[t4] - rv[t4]) +
                 c1 * ov[t4];
      }
    }
    bool big = false;
#pragma unroll
    for (int t4 = 0; t4 < 4; ++t4) {
      nv[t4] = up[t4] ? nv[t4] : ov[t4];
      big |= up[t4] && !(fabsf(nv[t4] - ov[t4]) < dmax_f) && nv[t4] != ov[t4];
    }
    const long rowo = ((long)k * cY + j) * cPQ;
    if (p < n) *reinterpret_cast<float4 *>(cL + COLOUR * cCS + rowo + q) = make_float4(nv[0], nv[1], nv[2], nv[3]);
    if (__any_sync(0xffffffffu, big)) {
#pragma unroll
      for (int t4 = 0; t4 < 4; ++t4) {
        const double d = fabs((double)nv[t4] - (double)ov[t4]);
        if (up[t4] && (d > dmax || d != d)) dmax = d;
      }
      dmax = warp_max_d(dmax);
      dmax_f = __double2float_rd(dmax);
    }
    if (COLOUR == 1 && k == 1) {
      // ground mirror of this span, both colours: red (j, 0) <- black (j, 1)
      // (the values just computed), black (j, 0) <- red (j, 1) (the stage's
      // other-colour row), for every cell of the row, updated or not
      const int qn = (cX + 1) >> 1;
      const long r0 = 0 * cCS + (long)j * cPQ, b0 = 1 * cCS + (long)j * cPQ;
      const float xcv[4] = {xc.x, xc.y, xc.z, xc.w};
#pragma unroll
      for (int t4 = 0; t4 < 4; ++t4) {
        if (p + t4 < n && q + t4 < qn) {
          cL[r0 + q + t4] = nv[t4];
          cL[b0 + q + t4] = xcv[t4];
        }
      }
    }
    __syncwarp();  // every lane is done with stage s before it is refilled
    if (issued < count) {
      if (!ASYNC && lane == 0) umma::fence_smem_async();
      issue(s);
      ++issued;
    } else if (ASYNC) {
      lane_commit();  // keep one group per iteration so wait_group<NS-1> stays exact
    }
  }
  if (ASYNC) lane_wait<0>();
  sweep_flush_end<MULTI>(dmax, MULTI ? (cerr ? cerr + cit : nullptr) : b.one.err + b.one.st->it);

  if (COLOUR == 1) sweep_finish_black<kUnitSpan, MULTI>(b, na);
}

}  // namespace qesb
