// Fused multi-sweep red-black SOR on the packed wall mask (the solver's hot
// kernel). Included by qesb_solver.cu, so it is compiled with -fmad=false and
// each cell update rounds exactly as Solver_CPU_RB.cpp:118-125 does.
//
// Scheme (per CTA): one x-y tile of the domain, marched bottom to top through
// every z plane. The tile owns TX x TY cells and loads a halo of H = 2K cells
// on each side (x rounded up to 16-byte rows), so K whole iterations (2K
// red/black half-steps) can run without hearing from neighbouring tiles:
// each half-step leaves one more ring of the halo stale. Along z the half-steps
// form a wavefront: at step s plane s is loaded and half-step h is applied to
// plane s-1-h, so when half-step h touches plane p, plane p+1 has just had
// half-step h-1 and plane p-1 still holds it (the red-black dependency order of
// one in-place sweep). A ring of W = 2K+2 planes lives in shared memory; the
// next plane is fetched into registers while the current step computes.
// Plane p is final, and written to the output buffer, after half-step 2K-1.
//
// Shared-memory planes use a red/black split row layout: row r holds the
// even-x cells in [0, BX/2) and the odd-x cells in [BX/2, BX). All cells one
// half-step updates sit in the same half, their x-neighbours in the other,
// so a warp's loads and stores hit 32 consecutive words.
//
// The ground mirror lambda(k=0) <- lambda(k=1) (Solver_CPU_RB.cpp:155-162) is
// applied in the ring after plane 1's black half-step of every iteration.
// Each iteration's max|dlambda| over the tile's own cells is kept in FP64
// and folded into err[] with one atomic per CTA and iteration.
#pragma once
#include "qesb_device.cuh"

namespace qesb {

struct TiledArgs {
  DevGrid G;
  const float *lam_in;
  float *lam_out;
  const float *R;
  const uint8_t *mask;
  const float *val;  // [6][Z] per-layer coefficient values e f g h m n
  const float *inv;  // [Z][64] omega / sum for each 6-bit wall mask
  double *err;       // per-iteration max|dlambda|
  SolveState *st;
  int itermax;
  int redo;          // 1: re-run st->redo iterations from st->redo_t0 (exact stop)
};

template <int K, int BX, int BY, int NT>
struct TileCfg {
  static constexpr int H = 2 * K;                 // halo cells (y)
  static constexpr int HX = (H + 3) / 4 * 4;      // halo cells (x), 16-byte aligned rows
  static constexpr int TX = BX - 2 * HX;
  static constexpr int TY = BY - 2 * H;
  static constexpr int W = 2 * K + 2;             // planes in the ring
  static constexpr int HB = BX / 2;               // half-row length
  static constexpr int CELLS = BX * BY;
  static constexpr int CHUNKS = CELLS / 4;        // 4-cell chunks per plane
  static constexpr int CPT = (CHUNKS + NT - 1) / NT;
  static constexpr int TAB = 72;                  // per-plane table: val[6] @0, inv[64] @8
  static constexpr size_t SMEM = (size_t)W * CELLS * (4 + 4 + 1) + (size_t)W * TAB * 4;
  static_assert(BX % 8 == 0 && TX > 0 && TY > 0, "tile too small for its halo");
  static_assert(HX <= kGX && H <= kGY, "halo exceeds the layout guards");
};

template <int K, int BX, int BY, int NT>
__global__ void __launch_bounds__(NT) k_sor_tiled(TiledArgs a)
{
  using C = TileCfg<K, BX, BY, NT>;
  extern __shared__ __align__(16) unsigned char smem[];
  float *sl = reinterpret_cast<float *>(smem);          // [W][BY][BX] lambda
  float *sr = sl + C::W * C::CELLS;                     // [W][BY][BX] R
  float *stab = sr + C::W * C::CELLS;                   // [W][TAB]
  uint8_t *sm = reinterpret_cast<uint8_t *>(stab + C::W * C::TAB);  // [W][BY][BX] mask

  SolveState *S = a.st;
  int t0, nit;
  if (a.redo) {
    t0 = S->redo_t0;
    nit = S->redo;
  } else {
    if (S->done) return;
    t0 = S->it;
    nit = min(K, a.itermax - t0);
  }
  if (nit <= 0) return;
  const int nh = 2 * nit;
  const DevGrid G = a.G;
  const int x0 = blockIdx.x * C::TX, y0 = blockIdx.y * C::TY;
  const int xs = x0 - C::HX, ys = y0 - C::H;
  const int tid = threadIdx.x;

  double emax[K];
#pragma unroll
  for (int t = 0; t < K; ++t) emax[t] = 0.0;

  float4 rl[C::CPT], rr[C::CPT];
  uint32_t rm[C::CPT];
  float rtab = 0.0f;

  auto gload = [&](int k) {
#pragma unroll
    for (int c = 0; c < C::CPT; ++c) {
      const int idx = tid + c * NT;
      if (idx < C::CHUNKS) {
        const int row = idx / (BX / 4), col = idx % (BX / 4);
        const long p = G.pad(xs + 4 * col, ys + row, k);
        rl[c] = __ldg(reinterpret_cast<const float4 *>(a.lam_in + p));
        rr[c] = __ldg(reinterpret_cast<const float4 *>(a.R + p));
        rm[c] = __ldg(reinterpret_cast<const uint32_t *>(a.mask + p));
      }
    }
    if (tid < C::TAB) {
      if (tid < 6) rtab = a.val[tid * G.Z + k];
      else if (tid >= 8) rtab = a.inv[k * 64 + (tid - 8)];
    }
  };
  auto sstore = [&](int k) {
    const int slot = k % C::W;
#pragma unroll
    for (int c = 0; c < C::CPT; ++c) {
      const int idx = tid + c * NT;
      if (idx < C::CHUNKS) {
        const int row = idx / (BX / 4), col = idx % (BX / 4);
        const int base = slot * C::CELLS + row * BX + 2 * col;  // even half; odd half at +HB
        *reinterpret_cast<float2 *>(sl + base) = make_float2(rl[c].x, rl[c].z);
        *reinterpret_cast<float2 *>(sl + base + C::HB) = make_float2(rl[c].y, rl[c].w);
        *reinterpret_cast<float2 *>(sr + base) = make_float2(rr[c].x, rr[c].z);
        *reinterpret_cast<float2 *>(sr + base + C::HB) = make_float2(rr[c].y, rr[c].w);
        const uint32_t m = rm[c];
        *reinterpret_cast<uint16_t *>(sm + base) = (uint16_t)((m & 0xffu) | ((m >> 8) & 0xff00u));
        *reinterpret_cast<uint16_t *>(sm + base + C::HB) = (uint16_t)(((m >> 8) & 0xffu) | ((m >> 16) & 0xff00u));
      }
    }
    if (tid < C::TAB) stab[slot * C::TAB + tid] = rtab;
  };
  // Owned cells of plane k (clipped to the domain) to the output buffer, two
  // x-adjacent cells (one even, one odd) per thread.
  auto writeout = [&](int k) {
    const int slot = k % C::W;
    for (int idx = tid; idx < C::TY * (C::TX / 2); idx += NT) {
      const int r = idx / (C::TX / 2), c2 = idx % (C::TX / 2);
      const int j = y0 + r, i = x0 + 2 * c2;
      if (j < G.Y && i < G.X) {
        const int ly = j - ys, q = (i - xs) >> 1;
        const float ev = sl[slot * C::CELLS + ly * BX + q];
        const float od = sl[slot * C::CELLS + ly * BX + C::HB + q];
        float *dst = a.lam_out + G.pad(i, j, k);
        if (i + 1 < G.X) *reinterpret_cast<float2 *>(dst) = make_float2(ev, od);
        else dst[0] = ev;
      }
    }
  };

  gload(0);
  sstore(0);
  __syncthreads();
  const int last = G.Z - 2 + nh;
  for (int s = 0; s <= last; ++s) {
    const bool pre = s + 1 < G.Z;
    if (pre) gload(s + 1);
#pragma unroll
    for (int h = 0; h < 2 * K; ++h) {
      const int p = s - 1 - h;
      if (h < nh && p >= 1 && p <= G.Z - 2) {
        const int colour = h & 1;
        const int sp = (p % C::W) * C::CELLS, su = ((p + 1) % C::W) * C::CELLS,
                  sd = ((p - 1) % C::W) * C::CELLS;
        const float *tb = stab + (p % C::W) * C::TAB;
        const float ve = tb[0], vf = tb[1], vg = tb[2], vh = tb[3], vm = tb[4], vn = tb[5];
        const int ylo = max(y0 - C::H + h + 1, 1), yhi = min(y0 + C::TY + C::H - h - 1, G.Y - 1);
        const int xlo = max(x0 - C::H + h + 1, 1), xhi = min(x0 + C::TX + C::H - h - 1, G.X - 1);
        const int rows = yhi - ylo;
        for (int idx = tid; idx < rows * C::HB; idx += NT) {
          const int r = idx / C::HB, q = idx % C::HB;
          const int j = ylo + r;
          const int par = (colour + j + p) & 1;  // x parity of this row's active cells
          const int lx = 2 * q + par, i = xs + lx;
          if (i < xlo || i >= xhi) continue;
          const int row = (j - ys) * BX;
          const int me = row + par * C::HB + q;
          const int ot = row + (1 - par) * C::HB;  // x-neighbours' half
          const float old = sl[sp + me];
          const float lxm = sl[sp + ot + q - (1 - par)];
          const float lxp = sl[sp + ot + q + par];
          const float lym = sl[sp + me - BX];
          const float lyp = sl[sp + me + BX];
          const float lzm = sl[sd + me];
          const float lzp = sl[su + me];
          const unsigned mk = sm[sp + me] & 63u;  // 6-bit wall mask: tb index stays inside the table
          const float e = (mk & 1u) ? ve : 0.0f, f = (mk & 2u) ? vf : 0.0f;
          const float g = (mk & 4u) ? vg : 0.0f, hh = (mk & 8u) ? vh : 0.0f;
          const float m = (mk & 16u) ? vm : 0.0f, n = (mk & 32u) ? vn : 0.0f;
          const float nv = tb[8 + mk] * (e * lxp + f * lxm + g * lyp + hh * lym + m * lzp + n * lzm - sr[sp + me]) +
                           (1.0f - kOmega) * old;
          sl[sp + me] = nv;
          if (i >= x0 && i < x0 + C::TX && j >= y0 && j < y0 + C::TY) {
            const double d = fabs((double)nv - (double)old);
            if (d > emax[h >> 1] || d != d) emax[h >> 1] = d;  // NaN propagates
          }
        }
        __syncthreads();
      }
    }
    // ground mirror after plane 1's black half-step (h = s - 2, odd)
    const int h1 = s - 2;
    if (h1 >= 0 && h1 < nh && (h1 & 1)) {
      const float4 *src = reinterpret_cast<const float4 *>(sl + (1 % C::W) * C::CELLS);
      float4 *dst = reinterpret_cast<float4 *>(sl);
      for (int idx = tid; idx < C::CELLS / 4; idx += NT) dst[idx] = src[idx];
      __syncthreads();
    }
    const int pf = s - nh;
    if (pf >= 1 && pf <= G.Z - 2) writeout(pf);
    if (s == nh + 1) writeout(0);
    if (s == G.Z - 1) writeout(G.Z - 1);
    __syncthreads();
    if (pre) sstore(s + 1);
    __syncthreads();
  }
#pragma unroll
  for (int t = 0; t < K; ++t) {
    if (t < nit) block_max_to(a.err + t0 + t, emax[t]);
    __syncthreads();
  }
}

}  // namespace qesb
