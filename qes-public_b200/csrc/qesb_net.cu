// Learned warm start: tensor-core kernels (tcgen05, BF16 operands, FP32
// accumulation in TMEM) for the 3D-convolution network, and their C ABI.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mutex>
#include <map>
#include <tuple>

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "qesb.h"
#include "qesb_internal.h"
#include "qesb_umma.cuh"

using namespace qesb;

namespace {

constexpr uint32_t kWaitLimit = 1u << 26;  // mbarrier polls before a kernel gives up
int g_conv_path = 0;  // 0: z-marching kernel for every forward convolution it takes (concatenated and
                      // upsampled inputs, rows of 128, 64 or 32; three output planes per MMA up to 32
                      // output channels), else direct, else implicit GEMM; 1: implicit GEMM only;
                      // 2: direct kernel, else implicit GEMM; 3 / 4: z-marching for one 16-channel input
                      // only, 2 / 4 rows per CTA; 5: as 3 with a four-stage implicit GEMM; 6: as 0 with
                      // one output plane per MMA

// Byte offset of element (r, k) in a canonical no-swizzle tile with KC = 64
// columns of K and R rows (see qesb_umma.cuh).
__device__ __forceinline__ uint32_t off_kmajor(int r, int k)
{
  return (uint32_t)(((r >> 3) * 8 + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
__device__ __forceinline__ uint32_t off_mnmajor(int r, int k, int R)
{
  return (uint32_t)(((k >> 3) * (R >> 3) + (r >> 3)) * 128 + (k & 7) * 16 + (r & 7) * 2);
}

// Self-test GEMM: C[128 x N] = A[128 x K] * B[N x K]^T, one CTA of 128
// threads, K a multiple of 64, operands copied into shared memory in
// K-major or MN-major canonical layout (a_mn, b_mn), accumulator in TMEM.
// A is row-major [128][K] (a_mn = 0) or [K][128] (a_mn = 1); likewise B.
__global__ void __launch_bounds__(128) k_umma_selftest(const __nv_bfloat16 *__restrict__ A,
                                                       const __nv_bfloat16 *__restrict__ B, float *__restrict__ C,
                                                       int N, int K, int a_mn, int b_mn, int *err)
{
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t *sa = sm;              // 128 x 64 bf16 = 16 KB
  uint8_t *sb = sm + 16384;      // N x 64 bf16 <= 32 KB
  __shared__ __align__(8) uint64_t mbar;
  __shared__ __align__(8) uint64_t mdrain;  // completion of every issued MMA, after a wait gave up
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
  if (warp == 0) umma::tmem_alloc(&tmem_base, ncols);
  if (tid == 0) {
    umma::mbar_init(&mbar, 1);
    umma::mbar_init(&mdrain, 1);
    umma::fence_mbar_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = umma::idesc_bf16(128, N, a_mn, b_mn);
  bool ok = true;
  for (int kc = 0; kc < K / 64 && ok; ++kc) {
    for (int idx = tid; idx < 128 * 64; idx += 128) {
      const int r = idx / 64, k = idx % 64;
      const __nv_bfloat16 v = a_mn ? A[(size_t)(kc * 64 + k) * 128 + r] : A[(size_t)r * K + kc * 64 + k];
      *reinterpret_cast<__nv_bfloat16 *>(sa + (a_mn ? off_mnmajor(r, k, 128) : off_kmajor(r, k))) = v;
    }
    for (int idx = tid; idx < N * 64; idx += 128) {
      const int r = idx / 64, k = idx % 64;
      const __nv_bfloat16 v = b_mn ? B[(size_t)(kc * 64 + k) * N + r] : B[(size_t)r * K + kc * 64 + k];
      *reinterpret_cast<__nv_bfloat16 *>(sb + (b_mn ? off_mnmajor(r, k, N) : off_kmajor(r, k))) = v;
    }
    umma::fence_smem_async();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t a0 = umma::smem_u32(sa), b0 = umma::smem_u32(sb);
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const uint64_t ad = a_mn ? umma::desc(a0 + kk * 2 * (128 / 8) * 128, (128 / 8) * 128, 128)
                                 : umma::desc(a0 + kk * 256, 128, 1024);
        const uint64_t bd = b_mn ? umma::desc(b0 + kk * 2 * (N / 8) * 128, (N / 8) * 128, 128)
                                 : umma::desc(b0 + kk * 256, 128, 1024);
        umma::mma_bf16(tmem, ad, bd, idesc, (kc > 0 || kk > 0) ? 1u : 0u);
      }
      umma::mma_commit(&mbar);
    }
    ok = umma::mbar_wait(&mbar, kc & 1, kWaitLimit);
    umma::fence_after_sync();
    __syncthreads();
  }
  if (!ok) {
    if (lane == 0) atomicExch(err, 1);
    umma::mma_drain(&mdrain, tid == 0, kWaitLimit);
  } else {
    for (int c0 = 0; c0 < N; c0 += 8) {
      float v[8];
      umma::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      const int row = warp * 32 + lane;
#pragma unroll
      for (int i = 0; i < 8; ++i) C[(size_t)row * N + c0 + i] = v[i];
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, ncols);
  }
}

// ---------------------------------------------------------------------------
// 3x3x3 convolutions as implicit GEMMs on the tensor cores
// ---------------------------------------------------------------------------
// Activations are channels-last BF16: T[(z*H + y)*W + x][C], C a multiple of
// 16 (padding channels are zero). A convolution's input may be the channel
// concatenation of two tensors (x1 with c1 channels, x2 with c2), and x1 may
// be stored at half resolution and read through a x2 nearest upsampling.
struct ConvIn {
  const __nv_bfloat16 *x1;
  const __nv_bfloat16 *x2;
  int c1, c2;  // cin = c1 + c2
  int up1;     // x1 at (D/2, H/2, W/2)
};

struct ConvGeom {
  int D, H, W;  // voxel grid of the GEMM rows (output grid)
  long V;       // D*H*W
  int Dc;       // depth of one item: D / Dc grids stacked along z, taps never cross from one to the next
};

// 16 bytes (8 channels c..c+7, never straddling x1/x2 since c1 % 16 == 0) of
// the input at voxel (z, y, x) for an output voxel at depth zo, or zeros
// outside the output voxel's item.
__device__ __forceinline__ uint4 load_in8(const ConvIn &in, const ConvGeom &g, int zo, int z, int y, int x, int c)
{
  const int zb = zo - zo % g.Dc;
  if (z < zb || z >= zb + g.Dc || y < 0 || y >= g.H || x < 0 || x >= g.W) return make_uint4(0, 0, 0, 0);
  const __nv_bfloat16 *p;
  if (c < in.c1) {
    if (in.up1)
      p = in.x1 + ((((long)(z >> 1) * (g.H >> 1) + (y >> 1)) * (g.W >> 1) + (x >> 1)) * in.c1 + c);
    else
      p = in.x1 + ((((long)z * g.H + y) * g.W + x) * in.c1 + c);
  } else {
    p = in.x2 + ((((long)z * g.H + y) * g.W + x) * in.c2 + (c - in.c1));
  }
  return __ldg(reinterpret_cast<const uint4 *>(p));
}

// 16-byte asynchronous copy global -> shared; valid = false fills zeros and reads nothing.
__device__ __forceinline__ void cp16_zfill(void *dst, const void *src, bool valid)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(umma::smem_u32(dst)), "l"(src),
               "r"(valid ? 16 : 0)
               : "memory");
}

__device__ __forceinline__ void tap_offset(int t, int &dz, int &dy, int &dx)
{
  dz = t / 9 - 1;
  dy = (t / 3) % 3 - 1;
  dx = t % 3 - 1;
}

struct ConvOut {
  __nv_bfloat16 *y;       // [V][N] BF16 (nullable when yf is set)
  float *yf;              // [V][N] FP32 (nullable)
  const float *bias;      // [N] (nullable)
  int relu;               // ReLU in the epilogue
  const __nv_bfloat16 *mask;  // [V][N] (nullable): zero where mask <= 0 (gradient through a ReLU)
  float *acc;             // split-K: [split][V][N] FP32 partial sums, one slice per K split (plain
                          // stores), summed in split order by k_conv_finish with the epilogue
  int ch0 = 0;            // yf holds output channel 0 alone, FP32 [V] (the z-marching kernel and the sums)
};

// Y[v][n] = epilogue( sum_k A[v][k] * Bm[n][k] ), A the implicit im2col of
// the input at taps v + sign*offset(t), k = t*cin + c, Bm [N][Kp] K-major
// BF16 (Kp = roundup(27*cin, 64), zero-padded). One CTA of 128 threads per
// 128 voxels; a ring of NSTAGES shared-memory stages filled by asynchronous
// 16-byte copies (zero-filled outside the grid) NSTAGES - 2 K chunks ahead,
// so the gathers of the next chunks are in flight while chunk j's MMAs run;
// accumulator N FP32 columns of TMEM.
template <int N, int NSTAGES>
__global__ void __launch_bounds__(128) k_conv_igemm(ConvIn in, ConvGeom g, int sign, const __nv_bfloat16 *__restrict__ Bm,
                                                   int Kp, ConvOut out, int *err)
{
  // split-K (gridDim.y > 1, small grids): CTA y sums the K chunks [jb, je)
  // and stores its partial in slice y of out.acc; k_conv_finish adds the
  // slices in order and applies the epilogue (the same bits every run).
  constexpr uint32_t SA = 128 * 64 * 2, SB = N * 64 * 2, STAGE = SA + SB;
  constexpr int NS = NSTAGES, DIST = NS - 2;  // chunk c's copies go out DIST iterations before its MMAs
  constexpr uint32_t NCOLS = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ __align__(8) uint64_t mbar[NS];  // stage s: the MMAs of chunk c, c % NS == s
  __shared__ __align__(8) uint64_t mdrain;  // completion of every issued MMA, after a wait gave up
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cin = in.c1 + in.c2;
  const long m0 = (long)blockIdx.x * 128;
  if (warp == 0) umma::tmem_alloc(&tmem_base, NCOLS);
  if (tid == 0) {
    for (int q = 0; q < NS; ++q) umma::mbar_init(&mbar[q], 1);
    umma::mbar_init(&mdrain, 1);
    umma::fence_mbar_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = umma::idesc_bf16(128, N, 0, 0);

  // this thread's 8 rows (m = tid/8 + 16 i) and fixed k-group g = tid % 8
  const int g8 = tid & 7;
  int rz[8], ry[8], rx[8], rzb[8];
  long rvox[8];
  bool rv[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const long v = m0 + (tid >> 3) + 16 * i;
    rv[i] = v < g.V;
    const long vv = rv[i] ? v : 0;
    rvox[i] = vv;
    rx[i] = (int)(vv % g.W);
    ry[i] = (int)((vv / g.W) % g.H);
    rz[i] = (int)(vv / ((long)g.W * g.H));
    rzb[i] = rz[i] - rz[i] % g.Dc;  // the row's item starts at this depth
  }
  const int nk_all = Kp / 64, per = (nk_all + gridDim.y - 1) / gridDim.y;
  const int jb = blockIdx.y * per, je = min(nk_all, jb + per), nk = je > jb ? je - jb : 0;
  // this thread's copies of local chunk jl into its stage (one commit group, empty past the range)
  auto issue = [&](int jl) {
    if (jl < nk) {
      const int j = jb + jl;
      uint8_t *sa = sm + (jl % NS) * STAGE, *sb = sa + SA;
      // A: rows m = tid/8 + 16 i, k-group g8
      const int kk = j * 64 + 8 * g8;
      const int t = kk / cin, c = kk - t * cin;
      int dz = 0, dy = 0, dx = 0;
      if (t < 27) tap_offset(t, dz, dy, dx);
      dz *= sign;
      dy *= sign;
      dx *= sign;
      if (in.up1 && c < in.c1) {  // the upsampled input: the coarse voxel of each fine one
        const int Hc = g.H >> 1, Wc = g.W >> 1;
        const __nv_bfloat16 *tb = in.x1 + c;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int z = rz[i] + dz, y = ry[i] + dy, x = rx[i] + dx;
          const bool valid = rv[i] && t < 27 && z >= rzb[i] && z < rzb[i] + g.Dc && (unsigned)y < (unsigned)g.H &&
                             (unsigned)x < (unsigned)g.W;
          const long cv = ((long)(z >> 1) * Hc + (y >> 1)) * Wc + (x >> 1);
          cp16_zfill(sa + off_kmajor((tid >> 3) + 16 * i, 8 * g8), valid ? tb + cv * in.c1 : in.x1, valid);
        }
      } else {  // same-grid input: one voxel offset for the tap, bounds per row
        const long dv = ((long)dz * g.H + dy) * g.W + dx;
        const bool first = c < in.c1;
        const __nv_bfloat16 *tb = first ? in.x1 + c : in.x2 + (c - in.c1);
        const int cs = first ? in.c1 : in.c2;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int z = rz[i] + dz, y = ry[i] + dy, x = rx[i] + dx;
          const bool valid = rv[i] && t < 27 && z >= rzb[i] && z < rzb[i] + g.Dc && (unsigned)y < (unsigned)g.H &&
                             (unsigned)x < (unsigned)g.W;
          cp16_zfill(sa + off_kmajor((tid >> 3) + 16 * i, 8 * g8), valid ? tb + (rvox[i] + dv) * cs : in.x1, valid);
        }
      }
      // B: N rows x 8 k-groups
      for (int idx = tid; idx < N * 8; idx += 128) {
        const int n = idx >> 3, gg = idx & 7;
        cp16_zfill(sb + off_kmajor(n, 8 * gg), Bm + (long)n * Kp + j * 64 + 8 * gg, true);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  bool ok = true;
  for (int jl = 0; jl < DIST; ++jl) issue(jl);
  for (int jl = 0; jl < nk && ok; ++jl) {
    // refill the stage chunk jl + DIST - NS used (its MMAs were issued two iterations ago)
    const int c = jl + DIST - NS;
    if (c >= 0) ok = umma::mbar_wait(&mbar[c % NS], (c / NS) & 1, kWaitLimit);
    if (!ok) break;
    issue(jl + DIST);
    asm volatile("cp.async.wait_group %0;" ::"n"(DIST) : "memory");  // chunk jl's copies (this thread's) landed
    umma::fence_smem_async();
    __syncthreads();  // everyone's
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t a0 = umma::smem_u32(sm + (jl % NS) * STAGE), b0 = a0 + SA;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        umma::mma_bf16(tmem, umma::desc(a0 + kk * 256, 128, 1024), umma::desc(b0 + kk * 256, 128, 1024), idesc,
                       (jl > 0 || kk > 0) ? 1u : 0u);
      umma::mma_commit(&mbar[jl % NS]);
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");  // no copy outlives the CTA's shared memory
  if (ok && nk > 0) ok = umma::mbar_wait(&mbar[(nk - 1) % NS], ((nk - 1) / NS) & 1, kWaitLimit);
  umma::fence_after_sync();
  if (!ok) {
    if (lane == 0) atomicExch(err, 1);
    umma::mma_drain(&mdrain, tid == 0, kWaitLimit);
  } else if (out.acc) {
    const long v = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < N; c0 += 8) {
      float a[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // an empty K range contributes zeros
      if (nk > 0) umma::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, a);
      if (v < g.V) {
#pragma unroll
        for (int q = 0; q < 8; ++q) out.acc[((long)blockIdx.y * g.V + v) * N + c0 + q] = a[q];
      }
    }
  } else {
    const long v = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < N; c0 += 8) {
      float a[8];
      umma::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, a);
      if (v < g.V) {
        if (out.bias) {
#pragma unroll
          for (int q = 0; q < 8; ++q) a[q] += __ldg(out.bias + c0 + q);
        }
        if (out.relu) {
#pragma unroll
          for (int q = 0; q < 8; ++q) a[q] = fmaxf(a[q], 0.0f);
        }
        if (out.mask) {
          const uint4 mk = __ldg(reinterpret_cast<const uint4 *>(out.mask + v * N + c0));
          const __nv_bfloat16 *mb = reinterpret_cast<const __nv_bfloat16 *>(&mk);
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (!(__bfloat162float(mb[q]) > 0.0f)) a[q] = 0.0f;
        }
        if (out.yf) {
          float4 *dst = reinterpret_cast<float4 *>(out.yf + v * N + c0);
          dst[0] = make_float4(a[0], a[1], a[2], a[3]);
          dst[1] = make_float4(a[4], a[5], a[6], a[7]);
        } else {
          uint4 pk;
          __nv_bfloat162 *h2 = reinterpret_cast<__nv_bfloat162 *>(&pk);
#pragma unroll
          for (int q = 0; q < 4; ++q) h2[q] = __floats2bfloat162_rn(a[2 * q], a[2 * q + 1]);
          *reinterpret_cast<uint4 *>(out.y + v * N + c0) = pk;
        }
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, NCOLS);
  }
}

// Direct 3x3x3 convolution for grids whose x rows are multiples of 128
// voxels (the network's full- and half-resolution levels, where the implicit
// GEMM's per-tap gather dominates). A CTA owns 128 consecutive x positions of
// TY x TZ output rows; for each 16-channel slice of the input it stages the
// (TY+2) x (TZ+2) rows of 130 voxels around them once in shared memory
// (cp.async, zero-filled outside the grid), laid out as
//     byte ((cg * NR + r) * 130 + xi) * 16,   cg = channel group of 8,
// so that for every tap (dz, dy, dx) the 128 x 16 A operand of an output row
// is a canonical K-major tile starting at row r(z+dz, y+dy), voxel 1+dx, with
// SBO = 128 B (next 8 voxels) and LBO = NR*130*16 B (next channel group): the
// 27 taps are 27 descriptors into the same tile, no im2col copy. B (all 27
// taps of the slice) is staged next to it. One thread issues the
// 27 * TY * TZ MMAs per slice into TY * TZ accumulators of N FP32 columns of
// TMEM. sign = -1 flips the taps (input gradient with the transposed weights).
constexpr int kDirTY = 2, kDirTZ = 2, kDirNR = (kDirTY + 2) * (kDirTZ + 2), kDirXW = 130;


// Address of the 8 channels c..c+7 of the input at voxel (z, y, x) (caller
// checks the grid bounds).
__device__ __forceinline__ const __nv_bfloat16 *in_ptr8(const ConvIn &in, const ConvGeom &g, int z, int y, int x,
                                                        int c)
{
  if (c < in.c1) {
    if (in.up1) return in.x1 + ((((long)(z >> 1) * (g.H >> 1) + (y >> 1)) * (g.W >> 1) + (x >> 1)) * in.c1 + c);
    return in.x1 + ((((long)z * g.H + y) * g.W + x) * in.c1 + c);
  }
  return in.x2 + ((((long)z * g.H + y) * g.W + x) * in.c2 + (c - in.c1));
}

template <int N>
__global__ void __launch_bounds__(128) k_conv_direct(ConvIn in, ConvGeom g, int sign,
                                                    const __nv_bfloat16 *__restrict__ Bm, int Kp, ConvOut out,
                                                    int *err)
{
  constexpr int TY = kDirTY, TZ = kDirTZ, NR = kDirNR, XW = kDirXW, NACC = TY * TZ;
  constexpr uint32_t SA = NR * XW * 32, SB = 27 * N * 32;
  constexpr uint32_t NCOLS = NACC * N <= 32 ? 32 : NACC * N <= 64 ? 64 : NACC * N <= 128 ? 128 : NACC * N <= 256 ? 256 : 512;
  static_assert(NACC * N <= 512, "accumulators exceed TMEM");
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ __align__(8) uint64_t mdrain;  // completion of every issued MMA, after a wait gave up
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cin = in.c1 + in.c2, KC = cin / 16;
  const int x0 = blockIdx.x * 128, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
  const int zb = z0 - z0 % g.Dc;  // the tile's item (TZ divides Dc)
  if (warp == 0) umma::tmem_alloc(&tmem_base, NCOLS);
  if (tid == 0) {
    umma::mbar_init(&mbar, 1);
    umma::mbar_init(&mdrain, 1);
    umma::fence_mbar_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = umma::idesc_bf16(128, N, 0, 0);
  uint8_t *sa = sm, *sb = sm + SA;
  bool ok = true;
  for (int kc = 0; kc < KC && ok; ++kc) {
    if (kc > 0) ok = umma::mbar_wait(&mbar, (kc - 1) & 1, kWaitLimit);  // the slice's MMAs read sa, sb
    if (!ok) break;
    for (int idx = tid; idx < NR * XW * 2; idx += 128) {
      const int cg = idx / (NR * XW), rem = idx - cg * NR * XW;
      const int r = rem / XW, xi = rem - r * XW;
      const int zz = z0 - 1 + r / (TY + 2), yy = y0 - 1 + r % (TY + 2), xx = x0 - 1 + xi;
      const bool inside = zz >= zb && zz < zb + g.Dc && yy >= 0 && yy < g.H && xx >= 0 && xx < g.W;
      const __nv_bfloat16 *src = inside ? in_ptr8(in, g, zz, yy, xx, 16 * kc + 8 * cg) : in.x1;
      cp16_zfill(sa + ((cg * NR + r) * XW + xi) * 16, src, inside);
    }
    for (int idx = tid; idx < 27 * N * 2; idx += 128) {
      const int t = idx / (N * 2), rem = idx - t * N * 2, n = rem >> 1, kg = rem & 1;
      cp16_zfill(sb + t * N * 32 + (n >> 3) * 256 + kg * 128 + (n & 7) * 16,
                 Bm + (long)n * Kp + t * cin + 16 * kc + 8 * kg, true);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    umma::fence_smem_async();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t a0 = umma::smem_u32(sa), b0 = umma::smem_u32(sb);
      for (int a = 0; a < NACC; ++a) {
        const int zt = a / TY, yt = a % TY;
        for (int t = 0; t < 27; ++t) {
          int dz, dy, dx;
          tap_offset(t, dz, dy, dx);
          const int r = (zt + 1 + sign * dz) * (TY + 2) + (yt + 1 + sign * dy);
          const uint64_t ad = umma::desc(a0 + (uint32_t)(r * XW + 1 + sign * dx) * 16, NR * XW * 16, 128);
          const uint64_t bd = umma::desc(b0 + (uint32_t)(t * N * 32), 128, 256);
          umma::mma_bf16(tmem + (uint32_t)(a * N), ad, bd, idesc, (kc > 0 || t > 0) ? 1u : 0u);
        }
      }
      umma::mma_commit(&mbar);
    }
  }
  if (ok) ok = umma::mbar_wait(&mbar, (KC - 1) & 1, kWaitLimit);
  umma::fence_after_sync();
  if (!ok) {
    if (lane == 0) atomicExch(err, 1);
    umma::mma_drain(&mdrain, tid == 0, kWaitLimit);
  } else {
    const int x = x0 + warp * 32 + lane;
    for (int a = 0; a < NACC; ++a) {
      const int z = z0 + a / TY, y = y0 + a % TY;
      const bool valid = z < g.D && y < g.H && x < g.W;
      const long v = ((long)z * g.H + y) * g.W + x;
      for (int c0 = 0; c0 < N; c0 += 8) {
        float f[8];
        umma::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(a * N + c0), f);
        if (!valid) continue;
        if (out.bias) {
#pragma unroll
          for (int q = 0; q < 8; ++q) f[q] += __ldg(out.bias + c0 + q);
        }
        if (out.relu) {
#pragma unroll
          for (int q = 0; q < 8; ++q) f[q] = fmaxf(f[q], 0.0f);
        }
        if (out.mask) {
          const uint4 mk = __ldg(reinterpret_cast<const uint4 *>(out.mask + v * N + c0));
          const __nv_bfloat16 *mb = reinterpret_cast<const __nv_bfloat16 *>(&mk);
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (!(__bfloat162float(mb[q]) > 0.0f)) f[q] = 0.0f;
        }
        if (out.yf) {
          float4 *dst = reinterpret_cast<float4 *>(out.yf + v * N + c0);
          dst[0] = make_float4(f[0], f[1], f[2], f[3]);
          dst[1] = make_float4(f[4], f[5], f[6], f[7]);
        } else {
          uint4 pk;
          __nv_bfloat162 *h2 = reinterpret_cast<__nv_bfloat162 *>(&pk);
#pragma unroll
          for (int q = 0; q < 4; ++q) h2[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
          *reinterpret_cast<uint4 *>(out.y + v * N + c0) = pk;
        }
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, NCOLS);
  }
}

// z-marching direct convolution. A CTA owns XT consecutive x positions
// (XT = 128, or the whole row when W is 64 or 32) of TY output rows and
// marches along z through up to ZC output planes of one item. Each input
// plane of (TY + 2) rows x (XT + 2) voxels (the x and y halos) arrives once,
// by one tensor-map copy per group of 8 channels (zeros outside the grid),
// into a ring of NS plane slots laid out as
//     byte q * CGB + p * 16,   q = channel group, p = r * (XT + 2) + xi,
// i.e. the staged rows one after the other as one flat row of voxels. The
// output positions use the same flattening (output row r, column x at
// p = r * (XT + 2) + x), so tap (dz, dy, dx) of a window of 128 consecutive
// output positions starting at s is a canonical K-major 128 x 16 A operand
// starting at staged position s + (1 + dy) * (XT + 2) + 1 + dx of the slot of
// plane z + dz (SBO 128 B, LBO CGB; the next 16 channels 2 * CGB further).
// With XT = 128 a window is one output row (s = r * 130); with XT < 128 the
// windows tile the flattened rows (s = 128 c) and the positions that fall on
// halo columns (x >= XT) are computed and dropped. Taps reaching past the
// item's z faces are not issued (zero padding). The staged channels may come
// from two inputs (a concatenation): kg1 groups of x1, then kg - kg1 of x2.
//
// Six warps, each role on its own mbarriers so that copies, MMAs and the
// read-out of different planes overlap:
//  * warp 4, one lane: copies plane i into slot i % NS once the MMAs of the
//    step that last read the slot's previous plane have completed (empty);
//  * warp 5, one lane: for output plane t, once planes t - 1 .. t + 1 have
//    landed (full) and the read-out of plane t - 2 has left accumulator set
//    t % 2 (acce), issues the C windows' 27 x KS MMAs into that set, then
//    commits them to accf[t % 2] and to empty[slot of plane t - 1];
//  * warps 0-3 (their TMEM lanes): read plane t's accumulators out when
//    accf[t % 2] completes, free the set (acce), then bias, ReLU and stores
//    (or, for a convolution split over its input channels, plain FP32 stores
//    into the launch's slice of out.acc).
// Every wait is bounded and also ends when another role has given up; a CTA
// that gives up lets its copies and MMAs finish, flags *err and stops.
struct ZfIn {
  int kg1, kg;  // channel groups of 8 staged per plane: kg1 from x1, kg - kg1 from x2 (kg even)
  int ch1, ch2; // first staged channel of x1 / of x2
  int c1, cin;  // channels of x1 and of the concatenation (the weights' K index is tap * cin + channel)
  int ns;       // plane slots in the ring (>= 4)
  int up1;      // x1 is the coarse grid (D/2 x H/2 x W/2): its planes are staged and upsampled in the CTA
};

template <int XT, int TY>
struct Zf {
  static constexpr int RWD = XT + 2;                                 // staged voxels per row
  static constexpr int S = XT == 128 ? RWD : 128;                    // output positions between windows
  static constexpr int C = XT == 128 ? TY : (TY * RWD + 127) / 128;  // windows (128-row MMAs) per plane
  static constexpr int STAGED = (TY + 2) * RWD;                      // positions one copy writes
  static constexpr int READ = (C - 1) * S + 128 + 2 * RWD + 2;       // positions the windows' taps read
  static constexpr uint32_t CGB = ((STAGED > READ ? STAGED : READ) * 16 + 127) / 128 * 128;
  static constexpr uint32_t BOX_TX = (uint32_t)STAGED * 16;          // bytes of one channel group's copy
  static_assert(C <= 4, "at most four windows per plane");
};

// The coarse planes of an upsampled input (k_conv_zflat3, up1): rows and
// columns of the coarse grid under a tile's staged rows, bytes per channel group.
template <int XT, int TY>
struct ZfUp {
  static constexpr int CR = TY / 2 + 2, CC = XT / 2 + 2;
  static constexpr uint32_t CCB = ((uint32_t)CR * CC * 16 + 127) / 128 * 128;
  static constexpr uint32_t BOX_TX = (uint32_t)CR * CC * 16;
};

// Shared memory of a launch: ns plane slots of kg channel groups, the
// weights, and (upsampled input) two coarse plane slots of up_kg groups.
template <int N, int XT, int TY>
__host__ __device__ constexpr uint32_t zf_smem_bytes(int kg, int ns, int up_kg = 0)
{
  return (uint32_t)ns * (uint32_t)kg * Zf<XT, TY>::CGB + 27u * (uint32_t)(kg / 2) * N * 32u +
         2u * (uint32_t)up_kg * ZfUp<XT, TY>::CCB;
}

// Bounded wait that also gives up as soon as another role of the CTA has
// (*abort set); sets *abort itself when its own polls run out.
__device__ __forceinline__ bool zf_wait(uint64_t *bar, uint32_t parity, volatile int *abort)
{
  for (uint32_t n = 0; n < kWaitLimit / 64; ++n) {
    if (umma::mbar_wait(bar, parity, 64)) return true;
    if (*abort) return false;
  }
  *abort = 1;
  return false;
}

template <int N, int XT, int TY>
__global__ void __launch_bounds__(192, 1) k_conv_zflat(const __grid_constant__ CUtensorMap map1,
                                                       const __grid_constant__ CUtensorMap map2, ZfIn zi, ConvGeom g,
                                                       int ZC, const __nv_bfloat16 *__restrict__ Bm, int Kp,
                                                       ConvOut out, int slice, int *err)
{
  using Z = Zf<XT, TY>;
  constexpr int C = Z::C, RWD = Z::RWD;
  constexpr uint32_t CGB = Z::CGB;
  constexpr uint32_t NCOLS = 2 * C * N <= 32 ? 32 : 2 * C * N <= 64 ? 64 : 2 * C * N <= 128 ? 128 : 2 * C * N <= 256 ? 256 : 512;
  static_assert(2 * C * N <= 512, "two accumulator sets exceed the TMEM columns");
  constexpr int kMaxNS = 8;
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ __align__(8) uint64_t full[kMaxNS];   // slot s: the copies (or a plain arrival) of its current plane
  __shared__ __align__(8) uint64_t empty[kMaxNS];  // slot s: the MMAs that read its current plane last are done
  __shared__ __align__(8) uint64_t accf[2];        // accumulator set b: the MMAs of plane t, t % 2 == b, are done
  __shared__ __align__(8) uint64_t acce[2];        // accumulator set b: plane t's read-out is done (4 warps)
  __shared__ __align__(8) uint64_t mdrain;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag, n_issued, n_landed, n_mma;
  volatile int *abort = &abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int KG = zi.kg, KS = KG >> 1, NS = zi.ns;
  const uint32_t SLOT = (uint32_t)KG * CGB;
  const int nzc = (g.Dc + ZC - 1) / ZC;
  const int item = blockIdx.z / nzc, zlo = item * g.Dc, zhi = zlo + g.Dc;
  const int z0 = zlo + (blockIdx.z % nzc) * ZC, z1 = min(z0 + ZC, zhi), nz = z1 - z0;
  const int x0 = blockIdx.x * XT, y0 = blockIdx.y * TY;
  uint8_t *sb = sm + (uint32_t)NS * SLOT;
  if ((umma::smem_u32(sm) & 127u) || NS < 4 || NS > kMaxNS) {  // copies need 128-byte aligned slots
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  if (warp == 0) umma::tmem_alloc(&tmem_base, NCOLS);
  if (tid == 0) {
    for (int q = 0; q < NS; ++q) {
      umma::mbar_init(&full[q], 1);
      umma::mbar_init(&empty[q], 1);
    }
    for (int b = 0; b < 2; ++b) {
      umma::mbar_init(&accf[b], 1);
      umma::mbar_init(&acce[b], 4);
    }
    umma::mbar_init(&mdrain, 1);
    umma::fence_mbar_init();
    abort_flag = 0;
    n_issued = n_landed = n_mma = 0;
  }
  // the weights, canonical K-major blocks of N rows x 16 channels, block (ks, tap) at (ks * 27 + tap) * N * 32
  for (int idx = tid; idx < 27 * KS * N * 2; idx += 192) {
    const int blk = idx / (N * 2), rem = idx - blk * N * 2, n = rem >> 1, kl = rem & 1;
    const int ks = blk / 27, t = blk - ks * 27, q = 2 * ks + kl;
    const int cc = q < zi.kg1 ? zi.ch1 + 8 * q : zi.c1 + zi.ch2 + 8 * (q - zi.kg1);
    cp16_zfill(sb + blk * N * 32 + (n >> 3) * 256 + kl * 128 + (n & 7) * 16, Bm + (long)n * Kp + t * zi.cin + cc, true);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  umma::fence_smem_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;

  if (warp == 4) {
    // ---- producer: plane index i is z = z0 - 1 + i (i = 0 .. nz + 1); planes
    // outside the item get a plain arrival instead of copies
    if (lane == 0) {
      int i = 0;
      for (; i <= nz + 1; ++i) {
        const int s = i % NS, k = i / NS;
        if (k >= 1 && !zf_wait(&empty[s], (uint32_t)(k - 1) & 1u, abort)) break;
        const int z = z0 - 1 + i;
        if (z < zlo || z >= zhi) {
          umma::mbar_arrive(&full[s]);
        } else {
          umma::mbar_expect_tx(&full[s], (uint32_t)KG * Z::BOX_TX);
          uint8_t *dst = sm + (uint32_t)s * SLOT;
          for (int q = 0; q < zi.kg1; ++q)
            umma::tma_load4(dst + q * CGB, &map1, zi.ch1 + 8 * q, x0 - 1, y0 - 1, z, &full[s]);
          for (int q = zi.kg1; q < KG; ++q)
            umma::tma_load4(dst + q * CGB, &map2, zi.ch2 + 8 * (q - zi.kg1), x0 - 1, y0 - 1, z, &full[s]);
        }
      }
      n_issued = i;
    }
  } else if (warp == 5) {
    // ---- MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = umma::idesc_bf16(128, N, 0, 0);
      const uint32_t a0 = umma::smem_u32(sm), b0 = umma::smem_u32(sb);
      const uint64_t ad0 = umma::desc(a0, CGB, 128);  // tap (0, -1, -1), first K step, window 0, slot 0
      const uint64_t bd0 = umma::desc(b0, 128, 256);  // weights block (0, 0)
      int landed = 0, t = 0;
      for (; t < nz; ++t) {
        bool ok = true;
        for (; ok && landed <= t + 2; ++landed) ok = zf_wait(&full[landed % NS], (uint32_t)(landed / NS) & 1u, abort);
        if (ok && t >= 2) ok = zf_wait(&acce[t & 1], (uint32_t)((t - 2) >> 1) & 1u, abort);
        if (!ok) break;
        umma::fence_after_sync();
        const int z = z0 + t;
        uint64_t sofs[3];  // slot offsets of planes z - 1, z, z + 1 (16-byte units)
#pragma unroll
        for (int d = 0; d < 3; ++d) sofs[d] = (uint64_t)((t + d) % NS) * (SLOT >> 4);
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const uint32_t acc = tmem + (uint32_t)((t & 1) * C * N + c * N);
          const uint64_t adc = ad0 + (uint64_t)(c * Z::S);
          uint32_t accum = 0;
          for (int ks = 0; ks < KS; ++ks) {
            const uint64_t aks = adc + (uint64_t)ks * (2 * CGB >> 4), bks = bd0 + (uint64_t)(ks * 27 * N * 2);
#pragma unroll
            for (int dz = -1; dz <= 1; ++dz) {
              if (z + dz < zlo || z + dz >= zhi) continue;
              const uint64_t as = aks + sofs[dz + 1];
#pragma unroll
              for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                for (int dx = 0; dx < 3; ++dx) {
                  constexpr int kN2 = N * 2;  // one block of N x 16 weights, 16-byte units
                  umma::mma_bf16(acc, as + (uint64_t)(dy * RWD + dx),
                                 bks + (uint64_t)(((dz + 1) * 9 + dy * 3 + dx) * kN2), idesc, accum);
                  accum = 1;
                }
            }
          }
        }
        umma::mma_commit(&accf[t & 1]);
        // plane index t (z - 1) is read by no later step: free its slot if a later plane needs it
        if (t + NS <= nz + 1) umma::mma_commit(&empty[t % NS]);
      }
      n_landed = landed;
      n_mma = t;
    }
  } else {
    // ---- read-out: warps 0-3, TMEM lanes 32 warp .. 32 warp + 31
    const int ny = min(TY, g.H - y0);  // rows of this tile inside the grid
    constexpr int WB = C * N <= 64 ? C : 64 / N > 0 ? 64 / N : 1;  // windows per TMEM wait (<= 64 registers)
    for (int t = 0; t < nz; ++t) {
      if (!zf_wait(&accf[t & 1], (uint32_t)(t >> 1) & 1u, abort)) break;
      umma::fence_after_sync();
      const int z = z0 + t;
#pragma unroll
      for (int c = 0; c < C; c += WB) {
        uint32_t raw[WB][N];
#pragma unroll
        for (int w = 0; w < WB; ++w)
#pragma unroll
          for (int c0 = 0; c0 < N; c0 += 16)
            if (c + w < C)
              umma::tmem_ld16_async(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((t & 1) * C * N + (c + w) * N + c0),
                                    *reinterpret_cast<uint32_t(*)[16]>(&raw[w][c0]));
        umma::tmem_wait_ld();
        if (c + WB >= C) {  // this warp's lanes of set t % 2 are all read
          umma::fence_before_sync();
          if (lane == 0) umma::mbar_arrive(&acce[t & 1]);
        }
#pragma unroll
        for (int w = 0; w < WB; ++w) {
          if (c + w >= C) break;
          const int p = (c + w) * Z::S + warp * 32 + lane, r = p / RWD, x = p - r * RWD;
          if (r >= ny || x >= XT) continue;
          const long v = ((long)z * g.H + y0 + r) * g.W + x0 + x;
          if (slice >= 0) {  // FP32 partial sum of this launch's channels
            float4 *dst = reinterpret_cast<float4 *>(out.acc + ((long)slice * g.V + v) * N);
#pragma unroll
            for (int c0 = 0; c0 < N; c0 += 4)
              dst[c0 / 4] = make_float4(__uint_as_float(raw[w][c0]), __uint_as_float(raw[w][c0 + 1]),
                                        __uint_as_float(raw[w][c0 + 2]), __uint_as_float(raw[w][c0 + 3]));
            continue;
          }
#pragma unroll
          for (int c0 = 0; c0 < N; c0 += 8) {
            float f[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) f[q] = __uint_as_float(raw[w][c0 + q]);
            if (out.bias) {
#pragma unroll
              for (int q = 0; q < 8; ++q) f[q] += __ldg(out.bias + c0 + q);
            }
            if (out.relu) {
#pragma unroll
              for (int q = 0; q < 8; ++q) f[q] = fmaxf(f[q], 0.0f);
            }
            if (out.ch0) {
              if (c0 == 0) out.yf[v] = f[0];
            } else if (out.yf) {
              float4 *dst = reinterpret_cast<float4 *>(out.yf + v * N + c0);
              dst[0] = make_float4(f[0], f[1], f[2], f[3]);
              dst[1] = make_float4(f[4], f[5], f[6], f[7]);
            } else {
              uint4 pk;
              __nv_bfloat162 *h2 = reinterpret_cast<__nv_bfloat162 *>(&pk);
#pragma unroll
              for (int q = 0; q < 4; ++q) h2[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
              *reinterpret_cast<uint4 *>(out.y + v * N + c0) = pk;
            }
          }
        }
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (abort_flag) {
    // a wait gave up: let every issued copy land and every issued MMA finish before TMEM and the slots go
    if (tid == 0) atomicExch(err, 1);
    if (tid == 160) {  // the issuer's thread: its MMAs tracked by one more commit
      umma::mma_commit(&mdrain);
      umma::mbar_wait(&mdrain, 0, kWaitLimit);
      for (int i = n_landed; i < n_issued; ++i) umma::mbar_wait(&full[i % NS], (uint32_t)(i / NS) & 1u, kWaitLimit);
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
  }
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, NCOLS);
  }
}

// The same convolution with each input plane read once per tap (dy, dx): the
// MMAs march over input planes, and the one of input plane i and tap (dy, dx)
// multiplies its window by [W(dz=+1) | W(dz=0) | W(dz=-1)] (N = 3 x cout),
// adding into the accumulators of output planes i - 2, i - 1 and i at once
// (input plane index i is z = z0 - 1 + i, output index t is z = z0 + t). A
// window's operand then leaves shared memory 9 x KS times per output plane
// instead of 27 x KS, which bounds these small-N MMAs. The accumulators of an
// output live in a TMEM ring of R slots per window (slot t % R): output t is
// complete after input plane t + 2, is read out, and its slot is written again
// by output t + R. Where the three outputs' slots wrap around the ring, and on
// the first tap of a plane (whose newest output starts from zero, as do all
// three on the item's first plane), the MMA is split into pieces of 1 or 2
// outputs. Roles as in k_conv_zflat; each input plane is read by one step, so
// its slot is freed right after that step's MMAs.
template <int C, int N>
__host__ __device__ constexpr int zf3_ring()
{
  return C * 8 * N <= 256 ? 8 : C * 5 * N <= 256 ? 5 : C * 4 * N <= 256 ? 4 : C * 8 * N <= 512 ? 8 : C * 5 * N <= 512 ? 5 : 4;
}

template <int N, int XT, int TY>
__global__ void __launch_bounds__(192, 1) k_conv_zflat3(const __grid_constant__ CUtensorMap map1,
                                                        const __grid_constant__ CUtensorMap map2, ZfIn zi, ConvGeom g,
                                                        int ZC, const __nv_bfloat16 *__restrict__ Bm, int Kp,
                                                        ConvOut out, int slice, int *err)
{
  using Z = Zf<XT, TY>;
  constexpr int C = Z::C, RWD = Z::RWD, R = zf3_ring<C, N>();
  constexpr uint32_t CGB = Z::CGB;
  constexpr uint32_t NCOLS = C * R * N <= 32 ? 32 : C * R * N <= 64 ? 64 : C * R * N <= 128 ? 128 : C * R * N <= 256 ? 256 : 512;
  static_assert(C * R * N <= 512 && R >= 4, "the output ring exceeds the TMEM columns");
  constexpr int kMaxNS = 8;
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ __align__(8) uint64_t full[kMaxNS];   // plane slot s: the copies (or a plain arrival) of its plane
  __shared__ __align__(8) uint64_t empty[kMaxNS];  // plane slot s: the MMAs of its plane are done
  __shared__ __align__(8) uint64_t accf[8];        // ring slot r: output t (t % R == r) is complete
  __shared__ __align__(8) uint64_t acce[8];        // ring slot r: output t is read out (4 warps)
  __shared__ __align__(8) uint64_t cfull[2];       // coarse slot b: the copies of its coarse plane (up1)
  __shared__ __align__(8) uint64_t mdrain;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag, n_issued, n_landed;
  volatile int *abort = &abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int KG = zi.kg, KS = KG >> 1, NS = zi.ns;
  const uint32_t SLOT = (uint32_t)KG * CGB;
  const int nzc = (g.Dc + ZC - 1) / ZC;
  const int item = blockIdx.z / nzc, zlo = item * g.Dc, zhi = zlo + g.Dc;
  const int z0 = zlo + (blockIdx.z % nzc) * ZC, z1 = min(z0 + ZC, zhi), nz = z1 - z0;
  const int x0 = blockIdx.x * XT, y0 = blockIdx.y * TY;
  uint8_t *sb = sm + (uint32_t)NS * SLOT;
  if ((umma::smem_u32(sm) & 127u) || NS < 2 || NS > kMaxNS) {  // copies need 128-byte aligned slots
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  if (warp == 0) umma::tmem_alloc(&tmem_base, NCOLS);
  if (tid == 0) {
    for (int q = 0; q < NS; ++q) {
      umma::mbar_init(&full[q], 1);
      umma::mbar_init(&empty[q], 1);
    }
    for (int r = 0; r < R; ++r) {
      umma::mbar_init(&accf[r], 1);
      umma::mbar_init(&acce[r], 4);
    }
    umma::mbar_init(&cfull[0], 1);
    umma::mbar_init(&cfull[1], 1);
    umma::mbar_init(&mdrain, 1);
    umma::fence_mbar_init();
    abort_flag = 0;
    n_issued = n_landed = 0;
  }
  // the weights: block (ks, dy, dx) of 3N rows x 16 channels, rows p * N + n holding tap dz = 1 - p
  for (int idx = tid; idx < 27 * KS * N * 2; idx += 192) {
    const int blk = idx / (6 * N), rem = idx - blk * 6 * N, np = rem >> 1, kl = rem & 1;
    const int ks = blk / 9, yx = blk - ks * 9, part = np / N, n = np - part * N, q = 2 * ks + kl;
    const int t = (2 - part) * 9 + yx;  // tap (dz, dy, dx) = (1 - part, yx / 3 - 1, yx % 3 - 1)
    const int cc = q < zi.kg1 ? zi.ch1 + 8 * q : zi.c1 + zi.ch2 + 8 * (q - zi.kg1);
    cp16_zfill(sb + blk * 3 * N * 32 + (np >> 3) * 256 + kl * 128 + (np & 7) * 16, Bm + (long)n * Kp + t * zi.cin + cc,
               true);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  umma::fence_smem_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;

  if (warp == 4 && zi.up1) {
    // ---- producer with an upsampled x1 (the whole warp): each coarse plane under the tile arrives once
    // by tensor-map copies into one of two coarse slots, one coarse plane ahead; the lanes expand it
    // (nearest neighbour) into the x1 channel groups of the fine slots of both fine planes it covers,
    // then lane 0 adds the copies of x2's groups and the plane's arrival
    using U = ZfUp<XT, TY>;
    uint8_t *cbuf = sb + 27u * (uint32_t)KS * N * 32u;
    const int cx0 = x0 / 2 - 1, cy0 = (y0 + 1) / 2 - 1;  // first coarse column and row (floor of (v - 1) / 2)
    const int czlo = zlo / 2, czmax = min(zhi / 2 - 1, z1 / 2);
    unsigned cis[2] = {0u, 0u}, cwt[2] = {0u, 0u};  // coarse loads issued / waited per slot (lane 0)
    int cnext = 0, chave = -1;
    int i = 0;
    for (; i <= nz + 1; ++i) {
      const int s = i % NS, k = i / NS;
      bool ok = true;
      if (lane == 0 && k >= 1) ok = zf_wait(&empty[s], (uint32_t)(k - 1) & 1u, abort);
      if (!__shfl_sync(0xffffffffu, ok, 0)) break;
      const int z = z0 - 1 + i;
      if (z < zlo || z >= zhi) {
        if (lane == 0) umma::mbar_arrive(&full[s]);
        continue;
      }
      const int c = z / 2;  // z >= zlo >= 0
      if (c != chave) {
        if (lane == 0) {
          if (cnext < c) cnext = c;
          for (; cnext <= c + 1 && cnext <= czmax && cnext >= czlo; ++cnext) {  // this plane and the next
            const int b = cnext & 1;
            umma::mbar_expect_tx(&cfull[b], (uint32_t)zi.kg1 * U::BOX_TX);
            for (int q = 0; q < zi.kg1; ++q)
              umma::tma_load4(cbuf + ((uint32_t)b * zi.kg1 + q) * U::CCB, &map1, zi.ch1 + 8 * q, cx0, cy0, cnext,
                              &cfull[b]);
            ++cis[b];
          }
          ok = zf_wait(&cfull[c & 1], cwt[c & 1] & 1u, abort);
          ++cwt[c & 1];
        }
        if (!__shfl_sync(0xffffffffu, ok, 0)) break;
        chave = c;
      }
      const uint8_t *cb = cbuf + (uint32_t)(c & 1) * zi.kg1 * U::CCB;
      uint8_t *dst = sm + (uint32_t)s * SLOT;
      for (int q = 0; q < zi.kg1; ++q)
#pragma unroll
        for (int ry = 0; ry < TY + 2; ++ry) {
          // staged row ry is fine row y0 - 1 + ry, coarse row floor((y0 + ry - 1) / 2) - cy0; staged column
          // rx is fine column x0 - 1 + rx, coarse column (rx + 1) / 2 - (x0 even)
          const uint4 *crow = reinterpret_cast<const uint4 *>(cb + q * U::CCB) + ((y0 + ry + 1) / 2 - 1 - cy0) * U::CC;
          uint4 *frow = reinterpret_cast<uint4 *>(dst + q * CGB) + ry * RWD;
          for (int rx = lane; rx < RWD; rx += 32) frow[rx] = crow[(rx + 1) >> 1];
        }
      umma::fence_smem_async();  // the expanded groups to the MMAs, the coarse slot's reads before its refill
      __syncwarp();
      if (lane == 0) {
        if (KG > zi.kg1) {
          umma::mbar_expect_tx(&full[s], (uint32_t)(KG - zi.kg1) * Z::BOX_TX);
          for (int q = zi.kg1; q < KG; ++q)
            umma::tma_load4(dst + q * CGB, &map2, zi.ch2 + 8 * (q - zi.kg1), x0 - 1, y0 - 1, z, &full[s]);
        } else {
          umma::mbar_arrive(&full[s]);
        }
      }
    }
    if (lane == 0) {
      n_issued = i;
      if (*abort)  // let the coarse copies in flight land before the CTA's memory goes
        for (int b = 0; b < 2; ++b)
          for (; cwt[b] < cis[b]; ++cwt[b]) umma::mbar_wait(&cfull[b], cwt[b] & 1u, kWaitLimit);
    }
  } else if (warp == 4) {
    // ---- producer: plane i (i = 0 .. nz + 1) into slot i % NS; planes outside the item get a plain arrival
    if (lane == 0) {
      int i = 0;
      for (; i <= nz + 1; ++i) {
        const int s = i % NS, k = i / NS;
        if (k >= 1 && !zf_wait(&empty[s], (uint32_t)(k - 1) & 1u, abort)) break;
        const int z = z0 - 1 + i;
        if (z < zlo || z >= zhi) {
          umma::mbar_arrive(&full[s]);
        } else {
          umma::mbar_expect_tx(&full[s], (uint32_t)KG * Z::BOX_TX);
          uint8_t *dst = sm + (uint32_t)s * SLOT;
          for (int q = 0; q < zi.kg1; ++q)
            umma::tma_load4(dst + q * CGB, &map1, zi.ch1 + 8 * q, x0 - 1, y0 - 1, z, &full[s]);
          for (int q = zi.kg1; q < KG; ++q)
            umma::tma_load4(dst + q * CGB, &map2, zi.ch2 + 8 * (q - zi.kg1), x0 - 1, y0 - 1, z, &full[s]);
        }
      }
      n_issued = i;
    }
  } else if (warp == 5) {
    // ---- MMA issuer: one step per input plane
    if (lane == 0) {
      const uint32_t idesc1 = umma::idesc_bf16(128, N, 0, 0), idesc2 = umma::idesc_bf16(128, 2 * N, 0, 0),
                     idesc3 = umma::idesc_bf16(128, 3 * N, 0, 0);
      const uint32_t a0 = umma::smem_u32(sm), b0 = umma::smem_u32(sb);
      const uint64_t ad0 = umma::desc(a0, CGB, 128);  // tap (dy, dx) = (-1, -1), first K step, window 0, slot 0
      const uint64_t bd0 = umma::desc(b0, 128, 256);  // weights block (0, 0, 0), row 0
      int i = 0;
      for (; i <= nz + 1; ++i) {
        bool ok = zf_wait(&full[i % NS], (uint32_t)(i / NS) & 1u, abort);
        const int prev = i - R;  // the output that held output i's ring slot
        if (ok && prev >= 0 && prev < nz) ok = zf_wait(&acce[prev % R], (uint32_t)(prev / R) & 1u, abort);
        if (!ok) break;
        umma::fence_after_sync();
        const int z = z0 - 1 + i;
        if (z >= zlo && z < zhi) {
          const bool first_in_item = z == zlo;  // outputs i - 2, i - 1, i all start here
          // the step's pieces of consecutive outputs (part pa.. of i - 2, i - 1, i, at ring slot sl): split
          // where the ring wraps; on the first tap also before output i (which starts from zero there)
          const int s0 = ((i - 2) % R + R) % R, wr = s0 + 3 <= R ? 3 : R - s0;  // parts before the wrap
          int npo = 1, pao[2] = {0, wr}, lno[2] = {wr, 3 - wr}, slo[2] = {s0, 0};
          if (wr < 3) npo = 2;
          int npf = 0, paf[3], lnf[3], slf[3];
          uint32_t acf[3];
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            if (k >= npo) break;
            const int a = pao[k], e = a + lno[k];  // parts [a, e)
            if (!first_in_item && a < 2 && e == 3) {  // split before part 2
              paf[npf] = a, lnf[npf] = 2 - a, slf[npf] = slo[k], acf[npf] = 1u, ++npf;
              paf[npf] = 2, lnf[npf] = 1, slf[npf] = slo[k] + 2 - a, acf[npf] = 0u, ++npf;
            } else {
              paf[npf] = a, lnf[npf] = e - a, slf[npf] = slo[k], acf[npf] = first_in_item || a == 2 ? 0u : 1u, ++npf;
            }
          }
          const uint64_t as = ad0 + (uint64_t)((i % NS) * (SLOT >> 4));
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const uint64_t adc = as + (uint64_t)(c * Z::S);
            const uint32_t colc = tmem + (uint32_t)(c * R * N);
            for (int ks = 0; ks < KS; ++ks) {
              const uint64_t aks = adc + (uint64_t)ks * (2 * CGB >> 4);
              const uint64_t bks = bd0 + (uint64_t)(ks * 9 * 3 * N * 2);  // 16-byte units
#pragma unroll
              for (int yx = 0; yx < 9; ++yx) {
                constexpr int kN2 = N * 2;
                const uint64_t ad = aks + (uint64_t)((yx / 3) * RWD + yx % 3);
                const uint64_t bd = bks + (uint64_t)(yx * 3 * kN2);
                if (ks == 0 && yx == 0) {
#pragma unroll
                  for (int k = 0; k < 3; ++k)
                    if (k < npf)
                      umma::mma_bf16(colc + (uint32_t)(slf[k] * N), ad, bd + (uint64_t)(paf[k] * kN2),
                                     lnf[k] == 1 ? idesc1 : lnf[k] == 2 ? idesc2 : idesc3, acf[k]);
                } else {
#pragma unroll
                  for (int k = 0; k < 2; ++k)
                    if (k < npo)
                      umma::mma_bf16(colc + (uint32_t)(slo[k] * N), ad, bd + (uint64_t)(pao[k] * kN2),
                                     lno[k] == 1 ? idesc1 : lno[k] == 2 ? idesc2 : idesc3, 1u);
                }
              }
            }
          }
        }
        // plane i is read by no later step: free its slot if a later plane needs it
        if (i + NS <= nz + 1) umma::mma_commit(&empty[i % NS]);
        if (i - 2 >= 0 && i - 2 < nz) umma::mma_commit(&accf[(i - 2) % R]);  // output i - 2 is complete
      }
      n_landed = i;
    }
  } else {
    // ---- read-out: warps 0-3, TMEM lanes 32 warp .. 32 warp + 31
    const int ny = min(TY, g.H - y0);  // rows of this tile inside the grid
    constexpr int WB = C * N <= 64 ? C : 64 / N > 0 ? 64 / N : 1;  // windows per TMEM wait (<= 64 registers)
    for (int t = 0; t < nz; ++t) {
      if (!zf_wait(&accf[t % R], (uint32_t)(t / R) & 1u, abort)) break;
      umma::fence_after_sync();
      const int z = z0 + t;
#pragma unroll
      for (int c = 0; c < C; c += WB) {
        uint32_t raw[WB][N];
#pragma unroll
        for (int w = 0; w < WB; ++w)
#pragma unroll
          for (int c0 = 0; c0 < N; c0 += 16)
            if (c + w < C)
              umma::tmem_ld16_async(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((c + w) * R * N + (t % R) * N + c0),
                                    *reinterpret_cast<uint32_t(*)[16]>(&raw[w][c0]));
        umma::tmem_wait_ld();
        if (c + WB >= C) {  // this warp's lanes of output t are all read
          umma::fence_before_sync();
          if (lane == 0) umma::mbar_arrive(&acce[t % R]);
        }
#pragma unroll
        for (int w = 0; w < WB; ++w) {
          if (c + w >= C) break;
          const int p = (c + w) * Z::S + warp * 32 + lane, r = p / RWD, x = p - r * RWD;
          if (r >= ny || x >= XT) continue;
          const long v = ((long)z * g.H + y0 + r) * g.W + x0 + x;
          if (slice >= 0) {  // FP32 partial sum of this launch's channels
            float4 *dst = reinterpret_cast<float4 *>(out.acc + ((long)slice * g.V + v) * N);
#pragma unroll
            for (int c0 = 0; c0 < N; c0 += 4)
              dst[c0 / 4] = make_float4(__uint_as_float(raw[w][c0]), __uint_as_float(raw[w][c0 + 1]),
                                        __uint_as_float(raw[w][c0 + 2]), __uint_as_float(raw[w][c0 + 3]));
            continue;
          }
#pragma unroll
          for (int c0 = 0; c0 < N; c0 += 8) {
            float f[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) f[q] = __uint_as_float(raw[w][c0 + q]);
            if (out.bias) {
#pragma unroll
              for (int q = 0; q < 8; ++q) f[q] += __ldg(out.bias + c0 + q);
            }
            if (out.relu) {
#pragma unroll
              for (int q = 0; q < 8; ++q) f[q] = fmaxf(f[q], 0.0f);
            }
            if (out.ch0) {
              if (c0 == 0) out.yf[v] = f[0];
            } else if (out.yf) {
              float4 *dst = reinterpret_cast<float4 *>(out.yf + v * N + c0);
              dst[0] = make_float4(f[0], f[1], f[2], f[3]);
              dst[1] = make_float4(f[4], f[5], f[6], f[7]);
            } else {
              uint4 pk;
              __nv_bfloat162 *h2 = reinterpret_cast<__nv_bfloat162 *>(&pk);
#pragma unroll
              for (int q = 0; q < 4; ++q) h2[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
              *reinterpret_cast<uint4 *>(out.y + v * N + c0) = pk;
            }
          }
        }
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (abort_flag) {
    // a wait gave up: let every issued copy land and every issued MMA finish before TMEM and the slots go
    if (tid == 0) atomicExch(err, 1);
    if (tid == 160) {  // the issuer's thread: its MMAs tracked by one more commit
      umma::mma_commit(&mdrain);
      umma::mbar_wait(&mdrain, 0, kWaitLimit);
      for (int i = n_landed; i < n_issued; ++i) umma::mbar_wait(&full[i % NS], (uint32_t)(i / NS) & 1u, kWaitLimit);
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
  }
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, NCOLS);
  }
}

// Weight gradient: dW[t*cin + c][n] += sum_v X[v + off(t)][c] * dY[v][n] over
// this CTA's voxel range. M-tile = 128 rows of (t, c); K = voxels in chunks
// of 64; both operands MN-major (channels contiguous). Partial sums from the
// CTAs of a row tile meet in dW (FP32) by atomicAdd.
template <int N>
__global__ void __launch_bounds__(128) k_conv_wgrad(ConvIn in, ConvGeom g, const __nv_bfloat16 *__restrict__ dY,
                                                   long vchunk, float *__restrict__ dW, int *err)
{
  constexpr uint32_t SA = 128 * 64 * 2, SB = N * 64 * 2, STAGE = SA + SB;
  constexpr uint32_t NCOLS = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ __align__(8) uint64_t mdrain;  // completion of every issued MMA, after a wait gave up
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cin = in.c1 + in.c2;
  const int Mrows = 27 * cin;
  const int mt0 = blockIdx.x * 128;
  const long vb = (long)blockIdx.y * vchunk, ve = min(g.V, vb + vchunk);
  if (vb >= ve) return;
  if (warp == 0) umma::tmem_alloc(&tmem_base, NCOLS);
  if (tid == 0) {
    umma::mbar_init(&mbar[0], 1);
    umma::mbar_init(&mbar[1], 1);
    umma::mbar_init(&mdrain, 1);
    umma::fence_mbar_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = umma::idesc_bf16(128, N, 1, 1);
  // this thread: voxel column kv = tid % 64 of each chunk; row groups rg = tid/64 + 2 i
  const int kv = tid & 63;
  int tg[8], cg[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int m = mt0 + 8 * ((tid >> 6) + 2 * i);
    tg[i] = m < Mrows ? m / cin : 27;
    cg[i] = m < Mrows ? m - tg[i] * cin : 0;
  }
  const int nk = (int)((ve - vb + 63) / 64);
  bool ok = true;
  for (int j = 0; j < nk && ok; ++j) {
    const int s = j & 1;
    if (j >= 2) ok = umma::mbar_wait(&mbar[s], ((j - 2) >> 1) & 1, kWaitLimit);
    if (!ok) break;
    uint8_t *sa = sm + s * STAGE, *sb = sa + SA;
    const long v = vb + (long)j * 64 + kv;
    const bool vin = v < ve;
    const int x = vin ? (int)(v % g.W) : 0, y = vin ? (int)((v / g.W) % g.H) : 0,
              z = vin ? (int)(v / ((long)g.W * g.H)) : 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      uint4 val = make_uint4(0, 0, 0, 0);
      if (vin && tg[i] < 27) {
        int dz, dy, dx;
        tap_offset(tg[i], dz, dy, dx);
        val = load_in8(in, g, z, z + dz, y + dy, x + dx, cg[i]);
      }
      *reinterpret_cast<uint4 *>(sa + off_mnmajor(8 * ((tid >> 6) + 2 * i), kv, 128)) = val;
    }
    for (int idx = tid; idx < N / 8 * 64; idx += 128) {
      const int ng = idx >> 6, k = idx & 63;
      const long vv = vb + (long)j * 64 + k;
      uint4 val = make_uint4(0, 0, 0, 0);
      if (vv < ve) val = __ldg(reinterpret_cast<const uint4 *>(dY + vv * N + 8 * ng));
      *reinterpret_cast<uint4 *>(sb + off_mnmajor(8 * ng, k, N)) = val;
    }
    umma::fence_smem_async();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t a0 = umma::smem_u32(sa), b0 = umma::smem_u32(sb);
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        umma::mma_bf16(tmem, umma::desc(a0 + kk * 2 * 16 * 128, 16 * 128, 128),
                       umma::desc(b0 + kk * 2 * (N / 8) * 128, (N / 8) * 128, 128), idesc,
                       (j > 0 || kk > 0) ? 1u : 0u);
      umma::mma_commit(&mbar[s]);
    }
  }
  if (ok) ok = umma::mbar_wait(&mbar[(nk - 1) & 1], ((nk - 1) >> 1) & 1, kWaitLimit);
  umma::fence_after_sync();
  if (!ok) {
    if (lane == 0) atomicExch(err, 1);
    umma::mma_drain(&mdrain, tid == 0, kWaitLimit);
  } else {
    const int m = mt0 + warp * 32 + lane;
    for (int c0 = 0; c0 < N; c0 += 8) {
      float a[8];
      umma::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, a);
      if (m < Mrows) {
#pragma unroll
        for (int q = 0; q < 8; ++q) atomicAdd(dW + (long)m * N + c0 + q, a[q]);
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, NCOLS);
  }
}

// Epilogue of a split-K convolution: y = act(sum of the split slices in
// order + bias), as k_conv_igemm's.
__global__ void k_conv_finish(const float *__restrict__ acc, int split, long V, int N, ConvOut out)
{
  for (long i = threadIdx.x + (long)blockIdx.x * blockDim.x; i < V * N; i += (long)gridDim.x * blockDim.x) {
    float a = acc[i];
    for (int y = 1; y < split; ++y) a += acc[(long)y * V * N + i];
    if (out.bias) a += __ldg(out.bias + (int)(i & (N - 1)));
    if (out.relu) a = fmaxf(a, 0.0f);
    if (out.mask && !(__bfloat162float(out.mask[i]) > 0.0f)) a = 0.0f;
    if (out.ch0) {
      if ((i & (N - 1)) == 0) out.yf[i / N] = a;
    } else if (out.yf) {
      out.yf[i] = a;
    } else {
      out.y[i] = __float2bfloat16_rn(a);
    }
  }
}

// The same, four consecutive elements per thread (16-byte aligned outputs):
// the same sums in the same order.
__global__ void k_conv_finish4(const float *__restrict__ acc, int split, long V, int N, ConvOut out)
{
  const long n4 = V * N / 4, slice4 = V * N / 4;
  const float4 *a4 = reinterpret_cast<const float4 *>(acc);
  for (long i = threadIdx.x + (long)blockIdx.x * blockDim.x; i < n4; i += (long)gridDim.x * blockDim.x) {
    float4 a = a4[i];
    for (int y = 1; y < split; ++y) {
      const float4 b = a4[(long)y * slice4 + i];
      a.x += b.x;
      a.y += b.y;
      a.z += b.z;
      a.w += b.w;
    }
    float f[4] = {a.x, a.y, a.z, a.w};
    const int n0 = (int)((i * 4) & (N - 1));
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (out.bias) f[q] += __ldg(out.bias + n0 + q);
      if (out.relu) f[q] = fmaxf(f[q], 0.0f);
      if (out.mask && !(__bfloat162float(out.mask[i * 4 + q]) > 0.0f)) f[q] = 0.0f;
    }
    if (out.ch0) {
      if (n0 == 0) out.yf[i * 4 / N] = f[0];
    } else if (out.yf) {
      reinterpret_cast<float4 *>(out.yf)[i] = make_float4(f[0], f[1], f[2], f[3]);
    } else {
      uint2 pk;
      __nv_bfloat162 *h2 = reinterpret_cast<__nv_bfloat162 *>(&pk);
      h2[0] = __floats2bfloat162_rn(f[0], f[1]);
      h2[1] = __floats2bfloat162_rn(f[2], f[3]);
      reinterpret_cast<uint2 *>(out.y)[i] = pk;
    }
  }
}

void launch_finish(const float *acc, int split, long V, int N, const ConvOut &out, cudaStream_t s)
{
  const bool vec = out.ch0 || (out.yf ? reinterpret_cast<uintptr_t>(out.yf) % 16 == 0 : reinterpret_cast<uintptr_t>(out.y) % 8 == 0);
  const long total = vec ? V * N / 4 : V * N;
  const unsigned blocks = (unsigned)std::min<long>((total + 255) / 256, 148L * 16);
  if (vec) k_conv_finish4<<<blocks, 256, 0, s>>>(acc, split, V, N, out);
  else k_conv_finish<<<blocks, 256, 0, s>>>(acc, split, V, N, out);
}

// Scratch buffers of the convolutions, one per (kind, device, stream) so that
// convolutions on different streams never share one; grown on demand and
// kept for the process. Kinds: FP32 partial sums of split convolutions, the
// upsampled input on the output grid, a full head output whose channel 0 is
// taken.
enum { kScratchAcc = 0, kScratchUp = 1, kScratchHead = 2 };
struct ScratchBuf {
  void *p = nullptr;
  size_t cap = 0;
};
std::mutex g_scratch_mu;
std::map<std::tuple<int, int, cudaStream_t>, ScratchBuf> g_scratch;

qesb_status scratch_buffer(int kind, int dev, cudaStream_t s, size_t bytes, void **out)
{
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  ScratchBuf &b = g_scratch[{kind, dev, s}];
  if (b.cap < bytes) {
    if (b.p) {
      cudaStreamSynchronize(s);  // the old buffer may still be read by this stream's work
      cudaFree(b.p);
    }
    b.p = nullptr;
    b.cap = 0;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "conv scratch buffer: %s", cudaGetErrorString(e));
    b.cap = bytes;
  }
  *out = b.p;
  return QESB_OK;
}

qesb_status acc_buffer(int dev, cudaStream_t s, size_t need, float **out)
{
  void *p = nullptr;
  const qesb_status st = scratch_buffer(kScratchAcc, dev, s, need * sizeof(float), &p);
  *out = static_cast<float *>(p);
  return st;
}

template <int N>
qesb_status launch_conv(const ConvIn &in, const ConvGeom &g, int sign, const __nv_bfloat16 *Bm, int Kp,
                        const ConvOut &out, int *err, cudaStream_t s)
{
  // three stages (gathers one chunk ahead, three CTAs per SM at N = 32), or four (two ahead) on conv path 5
  const bool three = g_conv_path != 5;
  const int smem = (three ? 3 : 4) * (128 * 64 * 2 + N * 64 * 2);
  int dev = 0;
  cudaGetDevice(&dev);
  static bool attr[64][2] = {};
  if (!attr[dev & 63][three]) {
    cudaError_t e = three ? cudaFuncSetAttribute(k_conv_igemm<N, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)
                          : cudaFuncSetAttribute(k_conv_igemm<N, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "conv attr: %s", cudaGetErrorString(e));
    attr[dev & 63][three] = true;
  }
  const unsigned blocks = (unsigned)((g.V + 127) / 128);
  // Small grids (fewer CTAs than about two per SM): split the K chunks over
  // grid.y, at least 4 chunks per split, partial sums in FP32.
  const int nk = Kp / 64;
  int split = 1;
  if (blocks < 296) split = std::max(1, std::min((int)(296 / blocks), nk / 4));
  ConvOut o = out;
  if (split > 1) {  // every slice element is written by exactly one CTA: no clearing
    const size_t need = (size_t)split * g.V * N;
    const qesb_status st = acc_buffer(dev, s, need, &o.acc);
    if (st != QESB_OK) return st;
  }
  if (three) k_conv_igemm<N, 3><<<dim3(blocks, split), 128, smem, s>>>(in, g, sign, Bm, Kp, o, err);
  else k_conv_igemm<N, 4><<<dim3(blocks, split), 128, smem, s>>>(in, g, sign, Bm, Kp, o, err);
  if (split > 1) {
    launch_finish(o.acc, split, g.V, N, out, s);
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? QESB_OK : qesb_fail(QESB_ERR_CUDA, "conv launch: %s", cudaGetErrorString(e));
}


template <int N>
qesb_status launch_conv_direct(const ConvIn &in, const ConvGeom &g, int sign, const __nv_bfloat16 *Bm, int Kp,
                               const ConvOut &out, int *err, cudaStream_t s)
{
  constexpr int smem = kDirNR * kDirXW * 32 + 27 * N * 32;
  int dev = 0;
  cudaGetDevice(&dev);
  static bool attr[64] = {};
  if (!attr[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(k_conv_direct<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "conv attr: %s", cudaGetErrorString(e));
    attr[dev & 63] = true;
  }
  const dim3 grid(g.W / 128, (g.H + kDirTY - 1) / kDirTY, (g.D + kDirTZ - 1) / kDirTZ);
  k_conv_direct<N><<<grid, 128, smem, s>>>(in, g, sign, Bm, Kp, out, err);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? QESB_OK : qesb_fail(QESB_ERR_CUDA, "conv launch: %s", cudaGetErrorString(e));
}

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled()
{
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && p &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// An input as a 4-D tensor (channel, x, y, z over all items), boxes of 8
// channels x (XT + 2) voxels x (TY + 2) rows x 1 plane; zeros outside.
qesb_status zf_map(CUtensorMap *map, const __nv_bfloat16 *x, int c, const ConvGeom &g, int XT, int TY)
{
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return qesb_fail(QESB_ERR_CUDA, "cuTensorMapEncodeTiled not available");
  const cuuint64_t cb = (cuuint64_t)c * 2;
  const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)g.W, (cuuint64_t)g.H, (cuuint64_t)g.D};
  const cuuint64_t st[3] = {cb, (cuuint64_t)g.W * cb, (cuuint64_t)g.W * g.H * cb};
  const cuuint32_t box[4] = {8, (cuuint32_t)(XT + 2), (cuuint32_t)(TY + 2), 1}, one[4] = {1, 1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16 *>(x), dims, st, box, one,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return qesb_fail(QESB_ERR_CUDA, "conv tensor map: cuTensorMapEncodeTiled failed (%d)", (int)r);
  return QESB_OK;
}

// The coarse grid under an upsampled input (D/2 x H/2 x W/2, c channels),
// boxes of 8 channels x cc columns x cr rows x 1 plane; zeros outside.
qesb_status zf_map_coarse(CUtensorMap *map, const __nv_bfloat16 *x, int c, const ConvGeom &g, int cc, int cr)
{
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return qesb_fail(QESB_ERR_CUDA, "cuTensorMapEncodeTiled not available");
  const cuuint64_t cb = (cuuint64_t)c * 2, W2 = (cuuint64_t)g.W / 2, H2 = (cuuint64_t)g.H / 2;
  const cuuint64_t dims[4] = {(cuuint64_t)c, W2, H2, (cuuint64_t)g.D / 2};
  const cuuint64_t st[3] = {cb, W2 * cb, W2 * H2 * cb};
  const cuuint32_t box[4] = {8, (cuuint32_t)cc, (cuuint32_t)cr, 1}, one[4] = {1, 1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16 *>(x), dims, st, box, one,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return qesb_fail(QESB_ERR_CUDA, "conv tensor map: cuTensorMapEncodeTiled failed (%d)", (int)r);
  return QESB_OK;
}

int max_dyn_smem()
{
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v - 1024;  // room for the kernel's static shared memory
}

// Whether a launch shape runs k_conv_zflat3 (three output planes per MMA):
// up to 32 output channels, an output ring within 256 TMEM columns (two CTAs
// per SM stay possible; measured slower otherwise), the default conv path.
template <int N, int XT, int TY>
constexpr bool zf_three_ok()
{
  return N <= 32 && Zf<XT, TY>::C * zf3_ring<Zf<XT, TY>::C, (N <= 32 ? N : 16)>() * N <= 256;
}

template <int N, int XT, int TY>
bool zf_uses_three()
{
  return zf_three_ok<N, XT, TY>() && g_conv_path == 0;
}

// Launches (channel splits) the z-marching convolution needs for cin input
// channels: the fewest whose 16-channel K steps, shared out evenly, fit the
// shared memory; 0 when even one step does not fit.
template <int N, int XT, int TY>
int zf_splits(int cin)
{
  const int steps = cin / 16, lim = max_dyn_smem(), ns = zf_uses_three<N, XT, TY>() ? 3 : 4;
  for (int P = 1; P <= steps; ++P)
    if ((int)zf_smem_bytes<N, XT, TY>(2 * ((steps + P - 1) / P), ns) <= lim) return P;
  return 0;
}

// Nearest-neighbour x2 upsampling of a coarse grid (D/2 x H/2 x W/2, c
// channels) onto the output grid, 16 bytes (8 channels) per thread.
__global__ void k_up2(const __nv_bfloat16 *__restrict__ x, ConvGeom g, int c, __nv_bfloat16 *__restrict__ y)
{
  const int cg = c / 8, n = g.W * cg;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int xq = i / cg, q = i - xq * cg;
  for (long row = blockIdx.y; row < (long)g.D * g.H; row += gridDim.y) {
    const int zq = (int)(row / g.H), yq = (int)(row - (long)zq * g.H);
    const long cv = ((long)(zq >> 1) * (g.H >> 1) + (yq >> 1)) * (g.W >> 1) + (xq >> 1);
    reinterpret_cast<uint4 *>(y)[row * n + i] = __ldg(reinterpret_cast<const uint4 *>(x) + cv * cg + q);
  }
}

// z-marching convolution of x1 (c1 channels) concatenated with x2 (c2), both
// on the output grid. Split over its input channels when the weights and the
// plane ring do not fit one CTA's shared memory: each launch stores its FP32
// partial sums in its own slice, k_conv_finish adds them in launch order and
// applies the epilogue.
template <int N, int XT, int TY>
qesb_status launch_conv_zflat(const __nv_bfloat16 *x1, int c1, int up1, const __nv_bfloat16 *x2, int c2,
                              const ConvGeom &g, const __nv_bfloat16 *Bm, int Kp, const ConvOut &out, int *err,
                              cudaStream_t s)
{
  const int cin = c1 + c2, steps = cin / 16, P = zf_splits<N, XT, TY>(cin);
  if (P == 0) return qesb_fail(QESB_ERR_ARG, "qesb_conv3d: %d channels do not fit the z-marching kernel", cin);
  const int per = (steps + P - 1) / P;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // an upsampled x1: staged from the coarse grid and expanded in the CTA (three-plane kernel, unsplit,
  // with three plane slots and the coarse slots fitting), else first written on the output grid
  int up_kg = 0;
  if (up1) {
    if (zf_uses_three<N, XT, TY>() && P == 1 && (int)zf_smem_bytes<N, XT, TY>(2 * steps, 3, c1 / 8) <= max_dyn_smem()) {
      up_kg = c1 / 8;
    } else {
      void *u = nullptr;
      qesb_status st = scratch_buffer(kScratchUp, dev, s, (size_t)g.V * c1 * 2, &u);
      if (st != QESB_OK) return st;
      const int n = g.W * (c1 / 8);
      const dim3 grid((unsigned)((n + 255) / 256), (unsigned)std::min<long>((long)g.D * g.H, 65535L));
      k_up2<<<grid, 256, 0, s>>>(x1, g, c1, static_cast<__nv_bfloat16 *>(u));
      x1 = static_cast<const __nv_bfloat16 *>(u);
    }
  }
  // one output plane per MMA, or three (k_conv_zflat3; not on conv path 6)
  constexpr int C = Zf<XT, TY>::C;
  constexpr bool kThreeOk = zf_three_ok<N, XT, TY>();
  const bool three = zf_uses_three<N, XT, TY>();
  void (*kern)(CUtensorMap, CUtensorMap, ZfIn, ConvGeom, int, const __nv_bfloat16 *, int, ConvOut, int, int *) =
      k_conv_zflat<N, XT, TY>;
  if constexpr (kThreeOk)
    if (three) kern = k_conv_zflat3<N, XT, TY>;
  // TMEM columns one CTA allocates: a CTA that needs all 512 must have its SM alone
  constexpr int kCols3 = C * zf3_ring<C, (kThreeOk ? N : 16)>() * N, kCols1 = 2 * C * N;
  const bool whole_sm = (three ? kCols3 : kCols1) > 256;
  // plane slots: four when two CTAs fit an SM (three-plane kernel: three when four do not fit), else as
  // many as fit (at most eight)
  const int lim = max_dyn_smem();
  int ns = 4;
  if (three && (int)zf_smem_bytes<N, XT, TY>(2 * per, 4, up_kg) > lim) ns = 3;
  if (whole_sm || 2 * ((int)zf_smem_bytes<N, XT, TY>(2 * per, ns, up_kg) + 1024) > lim + 1024)
    while (ns < 8 && (int)zf_smem_bytes<N, XT, TY>(2 * per, ns + 1, up_kg) <= lim) ++ns;
  int need = (int)zf_smem_bytes<N, XT, TY>(2 * per, ns, up_kg);
  if (whole_sm) need = std::max(need, (lim + 1024) / 2 + 1024);  // keeps a second CTA off the SM
  static int attr[64][2] = {};  // dynamic shared memory allowed so far, per device and kernel
  if (attr[dev & 63][three] < need) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, need);
    if (e != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "conv attr: %s", cudaGetErrorString(e));
    attr[dev & 63][three] = need;
  }
  CUtensorMap map1, map2;
  qesb_status st = up_kg ? zf_map_coarse(&map1, x1, c1, g, XT / 2 + 2, TY / 2 + 2) : zf_map(&map1, x1, c1, g, XT, TY);
  if (st != QESB_OK) return st;
  map2 = map1;
  if (c2 && (st = zf_map(&map2, x2, c2, g, XT, TY)) != QESB_OK) return st;
  ConvOut o = out;
  if (P > 1 && (st = acc_buffer(dev, s, (size_t)P * g.V * N, &o.acc)) != QESB_OK) return st;
  // z chunks: the length that minimises waves x (planes per CTA + ~3 planes of pipeline fill and weights)
  const int per_sm = std::max(1, (max_dyn_smem() + 1024) / (need + 1024));
  const long xy = (long)(g.W / XT) * ((g.H + TY - 1) / TY), items = g.D / g.Dc, slots = (long)sms * per_sm;
  int zc = g.Dc;
  long best = -1;
  for (int c = g.Dc; c >= 2; c = (c + 1) / 2) {
    const long waves = (xy * items * ((g.Dc + c - 1) / c) + slots - 1) / slots, cost = waves * (c + 3);
    if (best < 0 || cost < best) best = cost, zc = c;
    if (c == 2) break;
  }
  const dim3 grid(g.W / XT, (g.H + TY - 1) / TY, (unsigned)(items * ((g.Dc + zc - 1) / zc)));
  for (int p = 0; p < P; ++p) {
    const int a = p * per, b = std::min(steps, a + per);  // K steps (16 channels) [a, b) of the concatenation
    ZfIn zi;
    zi.kg = 2 * (b - a);
    zi.kg1 = std::max(0, std::min(zi.kg, (c1 - 16 * a) / 8));
    zi.ch1 = std::min(16 * a, c1);
    zi.ch2 = std::max(0, 16 * a - c1);
    zi.c1 = c1;
    zi.cin = cin;
    zi.ns = ns;
    zi.up1 = up_kg > 0;
    int smem = (int)zf_smem_bytes<N, XT, TY>(zi.kg, ns, up_kg);
    if (whole_sm) smem = std::max(smem, (lim + 1024) / 2 + 1024);
    kern<<<grid, 192, smem, s>>>(map1, map2, zi, g, zc, Bm, Kp, o, P > 1 ? p : -1, err);
  }
  if (P > 1) {
    launch_finish(o.acc, P, g.V, N, out, s);
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? QESB_OK : qesb_fail(QESB_ERR_CUDA, "conv launch: %s", cudaGetErrorString(e));
}


template <int N>
qesb_status launch_wgrad(const ConvIn &in, const ConvGeom &g, const __nv_bfloat16 *dY, long vchunk, float *dW,
                         int *err, cudaStream_t s)
{
  constexpr int smem = 2 * (128 * 64 * 2 + N * 64 * 2);
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_conv_wgrad<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "wgrad attr: %s", cudaGetErrorString(e));
    attr = true;
  }
  const int cin = in.c1 + in.c2;
  const dim3 grid((unsigned)((27 * cin + 127) / 128), (unsigned)((g.V + vchunk - 1) / vchunk));
  k_conv_wgrad<N><<<grid, 128, smem, s>>>(in, g, dY, vchunk, dW, err);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? QESB_OK : qesb_fail(QESB_ERR_CUDA, "wgrad launch: %s", cudaGetErrorString(e));
}

}  // namespace

extern "C" qesb_status qesb_umma_selftest(const uint16_t *A, const uint16_t *B, float *C, int N, int K, int a_mn,
                                          int b_mn)
{
  if (!A || !B || !C || N < 16 || N > 256 || N % 16 || K < 64 || K % 64)
    return qesb_fail(QESB_ERR_ARG, "qesb_umma_selftest: N in [16,256] step 16, K a multiple of 64");
  __nv_bfloat16 *dA = nullptr, *dB = nullptr;
  float *dC = nullptr;
  int *dErr = nullptr;
  cudaError_t e = cudaMalloc(&dA, sizeof(uint16_t) * 128 * K);
  if (e == cudaSuccess) e = cudaMalloc(&dB, sizeof(uint16_t) * N * K);
  if (e == cudaSuccess) e = cudaMalloc(&dC, sizeof(float) * 128 * N);
  if (e == cudaSuccess) e = cudaMalloc(&dErr, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(dA, A, sizeof(uint16_t) * 128 * K, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dB, B, sizeof(uint16_t) * N * K, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dErr, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(dC, 0, sizeof(float) * 128 * N);
  const int smem = 16384 + 32768;
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_umma_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  int herr = 0;
  if (e == cudaSuccess) {
    k_umma_selftest<<<1, 128, smem>>>(dA, dB, dC, N, K, a_mn, b_mn, dErr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(C, dC, sizeof(float) * 128 * N, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&herr, dErr, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dC);
  cudaFree(dErr);
  if (e != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "qesb_umma_selftest: %s", cudaGetErrorString(e));
  if (herr) return qesb_fail(QESB_ERR_CUDA, "qesb_umma_selftest: MMA completion wait timed out");
  return QESB_OK;
}

// ---------------------------------------------------------------------------
// conv C ABI (device pointers)
// ---------------------------------------------------------------------------
namespace {
bool conv_args_ok(int c1, int c2, int N, int D, int H, int W, int up1)
{
  return c1 > 0 && c1 % 16 == 0 && c2 >= 0 && c2 % 16 == 0 && (N == 16 || N == 32 || N == 64 || N == 128) &&
         D > 0 && H > 0 && W > 0 && (!up1 || (D % 2 == 0 && H % 2 == 0 && W % 2 == 0));
}
}  // namespace

namespace {

// Output channel 0 of an FP32 [V][N] tensor.
__global__ void k_take_ch0(const float *__restrict__ src, int N, long V, float *__restrict__ dst)
{
  for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < V; v += (long)gridDim.x * blockDim.x)
    dst[v] = src[v * N];
}

qesb_status conv_items(const void *x1, int c1, int up1, const void *x2, int c2, int items, int D, int H, int W,
                       int sign, const void *Bm, int Kp, int N, void *y, void *yf, const float *bias, int relu,
                       const void *mask, int *err, void *stream, int ch0)
{
  if (!conv_args_ok(c1, c2, N, D, H, W, up1) || items < 1 || (items > 1 && D % 2) || !x1 || (c2 && !x2) ||
      !Bm || (!y && !yf) || !err || (sign != 1 && sign != -1) || Kp < 27 * (c1 + c2) || Kp % 64 ||
      (ch0 && (!yf || y)))
    return qesb_fail(QESB_ERR_ARG, "qesb_conv3d: bad arguments");
  ConvIn in{static_cast<const __nv_bfloat16 *>(x1), static_cast<const __nv_bfloat16 *>(x2), c1, c2, up1};
  ConvGeom g{items * D, H, W, (long)items * D * H * W, D};
  ConvOut o{static_cast<__nv_bfloat16 *>(y), static_cast<float *>(yf), bias, relu,
            static_cast<const __nv_bfloat16 *>(mask)};
  const auto *B = static_cast<const __nv_bfloat16 *>(Bm);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0;
  cudaGetDevice(&dev);
  const auto aligned = [](const void *p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; };
  const bool fwd = sign == 1 && !mask && aligned(x1) && (!c2 || aligned(x2));
  if (fwd && (g_conv_path == 0 || g_conv_path == 6) && N <= 64) {
    // the z-marching kernel: rows of 128 (two output rows per CTA, one when
    // the channels of two do not fit unsplit), or whole rows of 64 or 32
    int xt = 0, ty = 0;
    const int cin = c1 + c2;
    if (W % 128 == 0) {
      xt = 128;
      const int p2 = N == 16 ? zf_splits<16, 128, 2>(cin) : N == 32 ? zf_splits<32, 128, 2>(cin) : zf_splits<64, 128, 2>(cin);
      const int p1 = N == 16 ? zf_splits<16, 128, 1>(cin) : N == 32 ? zf_splits<32, 128, 1>(cin) : zf_splits<64, 128, 1>(cin);
      ty = p2 == 1 || p1 != 1 ? 2 : 1;
    } else if (W == 64) {
      xt = 64, ty = 4;  // (two rows per CTA with three output planes per MMA measured 10-20 % slower)
    } else if (W == 32) {
      xt = 32, ty = 8;
    }
    if (xt) {
      const __nv_bfloat16 *xa = in.x1, *xb = in.x2;
      o.ch0 = ch0;
#define QESB_ZF(NN, XT_, TY_) launch_conv_zflat<NN, XT_, TY_>(xa, c1, up1, xb, c2, g, B, Kp, o, err, s)
      if (xt == 128 && ty == 2) return N == 16 ? QESB_ZF(16, 128, 2) : N == 32 ? QESB_ZF(32, 128, 2) : QESB_ZF(64, 128, 2);
      if (xt == 128) return N == 16 ? QESB_ZF(16, 128, 1) : N == 32 ? QESB_ZF(32, 128, 1) : QESB_ZF(64, 128, 1);
      if (xt == 64) return N == 16 ? QESB_ZF(16, 64, 4) : N == 32 ? QESB_ZF(32, 64, 4) : QESB_ZF(64, 64, 4);
      return N == 16 ? QESB_ZF(16, 32, 8) : N == 32 ? QESB_ZF(32, 32, 8) : QESB_ZF(64, 32, 8);
#undef QESB_ZF
    }
  }
  float *full = nullptr;  // channel 0 alone from the other kernels: their full output first
  if (ch0) {
    void *p = nullptr;
    qesb_status st = scratch_buffer(kScratchHead, dev, s, (size_t)g.V * N * sizeof(float), &p);
    if (st != QESB_OK) return st;
    full = static_cast<float *>(p);
    o.yf = full;
  }
  auto others = [&]() -> qesb_status {
    // paths 3, 4, 5: the z-marching kernel for one 16-channel input only (4 rows per CTA on path 4, else 2)
    if (fwd && g_conv_path >= 3 && W % 128 == 0 && (N == 16 || N == 32) && c1 == 16 && c2 == 0 && !up1) {
      if (g_conv_path == 4)
        return N == 16 ? launch_conv_zflat<16, 128, 4>(in.x1, 16, 0, nullptr, 0, g, B, Kp, o, err, s)
                       : launch_conv_zflat<32, 128, 4>(in.x1, 16, 0, nullptr, 0, g, B, Kp, o, err, s);
      return N == 16 ? launch_conv_zflat<16, 128, 2>(in.x1, 16, 0, nullptr, 0, g, B, Kp, o, err, s)
                     : launch_conv_zflat<32, 128, 2>(in.x1, 16, 0, nullptr, 0, g, B, Kp, o, err, s);
    }
    if ((g_conv_path == 0 || g_conv_path >= 2) && W % 128 == 0 && (N == 16 || N == 32)) {
      if (N == 16) return launch_conv_direct<16>(in, g, sign, B, Kp, o, err, s);
      return launch_conv_direct<32>(in, g, sign, B, Kp, o, err, s);
    }
    switch (N) {
      case 16: return launch_conv<16>(in, g, sign, B, Kp, o, err, s);
      case 32: return launch_conv<32>(in, g, sign, B, Kp, o, err, s);
      case 64: return launch_conv<64>(in, g, sign, B, Kp, o, err, s);
      default: return launch_conv<128>(in, g, sign, B, Kp, o, err, s);
    }
  };
  const qesb_status st = others();
  if (st != QESB_OK || !ch0) return st;
  k_take_ch0<<<(unsigned)std::min<long>((g.V + 255) / 256, 148L * 16), 256, 0, s>>>(full, N, g.V, static_cast<float *>(yf));
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? QESB_OK : qesb_fail(QESB_ERR_CUDA, "conv launch: %s", cudaGetErrorString(e));
}

}  // namespace

extern "C" qesb_status qesb_conv3d_items(const void *x1, int c1, int up1, const void *x2, int c2, int items, int D,
                                         int H, int W, int sign, const void *Bm, int Kp, int N, void *y, void *yf,
                                         const float *bias, int relu, const void *mask, int *err, void *stream)
{
  return conv_items(x1, c1, up1, x2, c2, items, D, H, W, sign, Bm, Kp, N, y, yf, bias, relu, mask, err, stream, 0);
}

qesb_status qesb_conv3d_head(const void *x1, int c1, int items, int D, int H, int W, const void *Bm, int Kp, int N,
                             float *y0, const float *bias, int relu, int *err, void *stream)
{
  return conv_items(x1, c1, 0, nullptr, 0, items, D, H, W, 1, Bm, Kp, N, nullptr, y0, bias, relu, nullptr, err,
                    stream, 1);
}

extern "C" qesb_status qesb_conv3d(const void *x1, int c1, int up1, const void *x2, int c2, int D, int H, int W,
                                   int sign, const void *Bm, int Kp, int N, void *y, void *yf, const float *bias,
                                   int relu, const void *mask, int *err, void *stream)
{
  return qesb_conv3d_items(x1, c1, up1, x2, c2, 1, D, H, W, sign, Bm, Kp, N, y, yf, bias, relu, mask, err, stream);
}

extern "C" qesb_status qesb_net_set_conv_path(int path)
{
  if (path < 0 || path > 6) return qesb_fail(QESB_ERR_ARG, "qesb_net_set_conv_path: path must be in [0, 6]");
  g_conv_path = path;
  return QESB_OK;
}

extern "C" qesb_status qesb_conv3d_wgrad(const void *x1, int c1, int up1, const void *x2, int c2, int D, int H,
                                         int W, const void *dY, int N, long vchunk, float *dW, int *err, void *stream)
{
  if (!conv_args_ok(c1, c2, N, D, H, W, up1) || !x1 || (c2 && !x2) || !dY || !dW || !err || vchunk < 64)
    return qesb_fail(QESB_ERR_ARG, "qesb_conv3d_wgrad: bad arguments");
  ConvIn in{static_cast<const __nv_bfloat16 *>(x1), static_cast<const __nv_bfloat16 *>(x2), c1, c2, up1};
  ConvGeom g{D, H, W, (long)D * H * W, D};
  const auto *d = static_cast<const __nv_bfloat16 *>(dY);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (N) {
    case 16: return launch_wgrad<16>(in, g, d, vchunk, dW, err, s);
    case 32: return launch_wgrad<32>(in, g, d, vchunk, dW, err, s);
    case 64: return launch_wgrad<64>(in, g, d, vchunk, dW, err, s);
    default: return launch_wgrad<128>(in, g, d, vchunk, dW, err, s);
  }
}

// ---------------------------------------------------------------------------
// elementwise kernels of the warm-start network (memory-bound, grid-stride)
// ---------------------------------------------------------------------------
namespace {

inline unsigned gs_blocks(long n, int per = 256) { return (unsigned)std::min<long>((n + per - 1) / per, 148L * 32); }

// 2x2x2 average pooling: y[(D/2)(H/2)(W/2)][C] from x[D][H][W][C] (BF16).
__global__ void k_pool2(const __nv_bfloat16 *__restrict__ x, __nv_bfloat16 *__restrict__ y, int D, int H, int W, int C)
{
  const int d = D / 2, h = H / 2, w = W / 2;
  const long n = (long)d * h * w * C;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long v = i / C;
    const int xx = (int)(v % w), yy = (int)((v / w) % h), zz = (int)(v / ((long)w * h));
    float s = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long src = (((long)(2 * zz + (q >> 2)) * H + 2 * yy + ((q >> 1) & 1)) * W + 2 * xx + (q & 1)) * C + c;
      s += __bfloat162float(x[src]);
    }
    y[i] = __float2bfloat16_rn(s * 0.125f);
  }
}

// The same, one thread per output voxel and group of 8 channels (16-byte
// loads and stores; the same sums in the same order). One block row per
// output row (zz, yy).
__global__ void k_pool2v(const __nv_bfloat16 *__restrict__ x, __nv_bfloat16 *__restrict__ y, int D, int H, int W,
                         int C)
{
  const int h = H / 2, w = W / 2, cg = C / 8, n = w * cg;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int xx = i / cg, q8 = i - xx * cg;
  for (long row = blockIdx.y; row < (long)(D / 2) * h; row += gridDim.y) {
    const int zz = (int)(row / h), yy = (int)(row - (long)zz * h);
    float acc[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long src = (((long)(2 * zz + (q >> 2)) * H + 2 * yy + ((q >> 1) & 1)) * W + 2 * xx + (q & 1)) * C + 8 * q8;
      const uint4 v = __ldg(reinterpret_cast<const uint4 *>(x + src));
      const __nv_bfloat162 *b2 = reinterpret_cast<const __nv_bfloat162 *>(&v);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float2 f = __bfloat1622float2(b2[e]);
        acc[2 * e] += f.x;
        acc[2 * e + 1] += f.y;
      }
    }
    uint4 pk;
    __nv_bfloat162 *o2 = reinterpret_cast<__nv_bfloat162 *>(&pk);
#pragma unroll
    for (int e = 0; e < 4; ++e) o2[e] = __floats2bfloat162_rn(acc[2 * e] * 0.125f, acc[2 * e + 1] * 0.125f);
    *reinterpret_cast<uint4 *>(y + (row * w + xx) * C + 8 * q8) = pk;
  }
}

// 2x2x2 average of an FP32 scalar field (training targets and weights of a
// network run at half resolution).
__global__ void k_pool2_f32(const float *__restrict__ x, float *__restrict__ y, int D, int H, int W)
{
  const int d = D / 2, h = H / 2, w = W / 2;
  const long n = (long)d * h * w;
  for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < n; v += (long)gridDim.x * blockDim.x) {
    const int xx = (int)(v % w), yy = (int)((v / w) % h), zz = (int)(v / ((long)w * h));
    float s = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q)
      s += x[((long)(2 * zz + (q >> 2)) * H + 2 * yy + ((q >> 1) & 1)) * W + 2 * xx + (q & 1)];
    y[v] = s * 0.125f;
  }
}

// Gradient into a skip tensor e (level grid D x H x W, C channels):
//   g_e = (gcat[v][coff + c] + gpool[parent(v)][c] / 8) * (e[v][c] > 0)
// gcat: FP32 input gradient of the decoder conv that reads e (its channels
// coff.. coff+C-1); gpool: FP32 gradient of pool(e) (nullable).
__global__ void k_skip_grad(const float *__restrict__ gcat, int ccat, int coff, const float *__restrict__ gpool,
                            const __nv_bfloat16 *__restrict__ e, __nv_bfloat16 *__restrict__ ge, int D, int H, int W,
                            int C)
{
  const long n = (long)D * H * W * C;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long v = i / C;
    float g = gcat[v * ccat + coff + c];
    if (gpool) {
      const int x = (int)(v % W), y = (int)((v / W) % H), z = (int)(v / ((long)W * H));
      g += gpool[((((long)(z >> 1) * (H >> 1)) + (y >> 1)) * (W >> 1) + (x >> 1)) * C + c] * 0.125f;
    }
    ge[i] = __float2bfloat16_rn(__bfloat162float(e[i]) > 0.0f ? g : 0.0f);
  }
}

// Gradient of an upsampled input: gx[vlow][c] = sum over the 8 children of
// gcat[child][c] (channels 0..C-1 of gcat), times (x[vlow][c] > 0).
__global__ void k_up_grad(const float *__restrict__ gcat, int ccat, const __nv_bfloat16 *__restrict__ x,
                          __nv_bfloat16 *__restrict__ gx, int D, int H, int W, int C)
{
  const int d = D / 2, h = H / 2, w = W / 2;
  const long n = (long)d * h * w * C;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long v = i / C;
    const int xx = (int)(v % w), yy = (int)((v / w) % h), zz = (int)(v / ((long)w * h));
    float s = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q)
      s += gcat[(((long)(2 * zz + (q >> 2)) * H + 2 * yy + ((q >> 1) & 1)) * W + 2 * xx + (q & 1)) * ccat + c];
    gx[i] = __float2bfloat16_rn(__bfloat162float(x[i]) > 0.0f ? s : 0.0f);
  }
}

// FP32 -> BF16 with an optional ReLU-derivative mask (same shape).
__global__ void k_to_bf16_masked(const float *__restrict__ g, const __nv_bfloat16 *__restrict__ mask,
                                 __nv_bfloat16 *__restrict__ out, long n)
{
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float v = g[i];
    out[i] = __float2bfloat16_rn(!mask || __bfloat162float(mask[i]) > 0.0f ? v : 0.0f);
  }
}

// Column sums db[c] += sum_v g[v][c] (BF16 gradient), per-block partials.
__global__ void k_colsum(const __nv_bfloat16 *__restrict__ g, long V, int C, float *__restrict__ db)
{
  extern __shared__ float part[];
  for (int c = threadIdx.x; c < C; c += blockDim.x) part[c] = 0.0f;
  __syncthreads();
  const int lanes = blockDim.x / C * C;  // threads grouped by channel
  if ((int)threadIdx.x < lanes) {
    const int c = threadIdx.x % C;
    float s = 0.0f;
    for (long v = blockIdx.x * (long)(lanes / C) + threadIdx.x / C; v < V; v += (long)gridDim.x * (lanes / C))
      s += __bfloat162float(g[v * C + c]);
    atomicAdd(&part[c], s);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(&db[c], part[c]);
}

// Loss over valid cells: pred = yhead[v][0] (FP32, head channel stride N),
// L += sum ((pred - tgt) w[v])^2 / count; gradient 2 (pred - tgt) w / count
// into channel 0 of g (BF16 [V][N], other channels zero).
__global__ void k_mse(const float *__restrict__ yhead, int N, const float *__restrict__ tgt,
                      const float *__restrict__ w, long V, float inv_count, __nv_bfloat16 *__restrict__ g,
                      double *__restrict__ loss)
{
  double acc = 0.0;
  for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < V; v += (long)gridDim.x * blockDim.x) {
    const float d = (yhead[v * N] - tgt[v]) * w[v];
    acc += (double)d * d * inv_count;
    g[v * N] = __float2bfloat16_rn(2.0f * d * inv_count);
    for (int c = 1; c < N; ++c) g[v * N + c] = __float2bfloat16_rn(0.0f);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

// Low-frequency loss term: the error e = (pred - tgt) w averaged over F x F x F
// blocks (one thread per block), E_c; loss += beta * sum_c E_c^2 / nc and
// g[v][0] += 2 beta E_c w[v] / (F^3 nc) on the block's cells. Weights the
// smooth part of the error, which red-black SOR removes slowest.
__global__ void k_mse_coarse(const float *__restrict__ yhead, int N, const float *__restrict__ tgt,
                             const float *__restrict__ w, int D, int H, int W, int F, float beta,
                             __nv_bfloat16 *__restrict__ g, double *__restrict__ loss)
{
  const int d = D / F, h = H / F, ww = W / F;
  const long nc = (long)d * h * ww;
  const float f3 = (float)(F * F * F);
  double acc = 0.0;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < nc; c += (long)gridDim.x * blockDim.x) {
    const int cx = (int)(c % ww), cy = (int)((c / ww) % h), cz = (int)(c / ((long)ww * h));
    float e = 0.0f;
    for (int q = 0; q < F * F * F; ++q) {
      const long v = ((long)(cz * F + q / (F * F)) * H + cy * F + (q / F) % F) * W + cx * F + q % F;
      e += (yhead[v * N] - tgt[v]) * w[v];
    }
    e /= f3;
    acc += (double)beta * e * e / (double)nc;
    const float gs = 2.0f * beta * e / (f3 * (float)nc);
    for (int q = 0; q < F * F * F; ++q) {
      const long v = ((long)(cz * F + q / (F * F)) * H + cy * F + (q / F) % F) * W + cx * F + q % F;
      g[v * N] = __float2bfloat16_rn(__bfloat162float(g[v * N]) + gs * w[v]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

// Adam on one conv layer (Kingma & Ba 2015): master weights W[27*cin][cout]
// (row t*cin + c), moments m, v, gradient dW; bias likewise. Writes the two
// BF16 GEMM layouts: Bm[cout][Kp] (k = t*cin + c) and Bd[cin][Kd] (k = t*cout + o).
__global__ void k_adam_conv(float *__restrict__ Wt, float *__restrict__ m, float *__restrict__ v,
                            const float *__restrict__ dW, int cin, int cout, int cout_real,
                            __nv_bfloat16 *__restrict__ Bm, int Kp, __nv_bfloat16 *__restrict__ Bd, int Kd,
                            float lr, float b1, float b2, float eps, float c1, float c2, float grad_scale)
{
  const long n = 27L * cin * cout;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int o = (int)(i % cout);
    const long row = i / cout;  // t*cin + c
    const int t = (int)(row / cin), c = (int)(row % cin);
    float w = Wt[i];
    if (o < cout_real) {
      const float g = dW[i] * grad_scale;
      const float mm = b1 * m[i] + (1.0f - b1) * g;
      const float vv = b2 * v[i] + (1.0f - b2) * g * g;
      m[i] = mm;
      v[i] = vv;
      w -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
      Wt[i] = w;
    }
    const __nv_bfloat16 wb = __float2bfloat16_rn(o < cout_real ? w : 0.0f);
    Bm[(long)o * Kp + row] = wb;
    if (Bd) Bd[(long)c * Kd + (long)t * cout + o] = wb;
  }
}

__global__ void k_adam_vec(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                           const float *__restrict__ g, int n, float lr, float b1, float b2, float eps, float c1,
                           float c2, float grad_scale)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const float gg = g[i] * grad_scale;
    const float mm = b1 * m[i] + (1.0f - b1) * gg;
    const float vv = b2 * v[i] + (1.0f - b2) * gg * gg;
    m[i] = mm;
    v[i] = vv;
    p[i] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  }
}

}  // namespace

#define NET_CK(expr)                                                                               \
  do {                                                                                             \
    cudaError_t e_ = (expr);                                                                       \
    if (e_ != cudaSuccess) return qesb_fail(QESB_ERR_CUDA, "%s: %s", __func__, cudaGetErrorString(e_)); \
  } while (0)

extern "C" {

qesb_status qesb_net_pool2(const void *x, void *y, int D, int H, int W, int C, void *stream)
{
  if (!x || !y || D % 2 || H % 2 || W % 2 || C <= 0) return qesb_fail(QESB_ERR_ARG, "qesb_net_pool2: bad arguments");
  if (C % 8 == 0 && reinterpret_cast<uintptr_t>(x) % 16 == 0 && reinterpret_cast<uintptr_t>(y) % 16 == 0) {
    const int n = (W / 2) * (C / 8);
    const dim3 grid((unsigned)((n + 127) / 128), (unsigned)std::min<long>((long)(D / 2) * (H / 2), 65535L));
    k_pool2v<<<grid, 128, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)x, (__nv_bfloat16 *)y, D, H, W, C);
  } else {
    const long n = (long)(D / 2) * (H / 2) * (W / 2) * C;
    k_pool2<<<gs_blocks(n), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)x, (__nv_bfloat16 *)y, D, H, W, C);
  }
  NET_CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_net_pool2_f32(const float *x, float *y, int D, int H, int W, void *stream)
{
  if (!x || !y || D % 2 || H % 2 || W % 2) return qesb_fail(QESB_ERR_ARG, "qesb_net_pool2_f32: bad arguments");
  const long n = (long)(D / 2) * (H / 2) * (W / 2);
  k_pool2_f32<<<gs_blocks(n), 256, 0, (cudaStream_t)stream>>>(x, y, D, H, W);
  NET_CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_net_skip_grad(const float *gcat, int ccat, int coff, const float *gpool, const void *e, void *ge,
                               int D, int H, int W, int C, void *stream)
{
  if (!gcat || !e || !ge || coff + C > ccat) return qesb_fail(QESB_ERR_ARG, "qesb_net_skip_grad: bad arguments");
  const long n = (long)D * H * W * C;
  k_skip_grad<<<gs_blocks(n), 256, 0, (cudaStream_t)stream>>>(gcat, ccat, coff, gpool, (const __nv_bfloat16 *)e,
                                                              (__nv_bfloat16 *)ge, D, H, W, C);
  NET_CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_net_up_grad(const float *gcat, int ccat, const void *x, void *gx, int D, int H, int W, int C,
                             void *stream)
{
  if (!gcat || !x || !gx || C > ccat || D % 2 || H % 2 || W % 2)
    return qesb_fail(QESB_ERR_ARG, "qesb_net_up_grad: bad arguments");
  const long n = (long)(D / 2) * (H / 2) * (W / 2) * C;
  k_up_grad<<<gs_blocks(n), 256, 0, (cudaStream_t)stream>>>(gcat, ccat, (const __nv_bfloat16 *)x, (__nv_bfloat16 *)gx,
                                                            D, H, W, C);
  NET_CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_net_to_bf16(const float *g, const void *mask, void *out, long n, void *stream)
{
  if (!g || !out || n <= 0) return qesb_fail(QESB_ERR_ARG, "qesb_net_to_bf16: bad arguments");
  k_to_bf16_masked<<<gs_blocks(n), 256, 0, (cudaStream_t)stream>>>(g, (const __nv_bfloat16 *)mask,
                                                                   (__nv_bfloat16 *)out, n);
  NET_CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_net_colsum(const void *g, long V, int C, float *db, void *stream)
{
  if (!g || !db || C <= 0 || C > 256) return qesb_fail(QESB_ERR_ARG, "qesb_net_colsum: bad arguments");
  k_colsum<<<148 * 4, 256, C * sizeof(float), (cudaStream_t)stream>>>((const __nv_bfloat16 *)g, V, C, db);
  NET_CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_net_mse(const float *yhead, int N, const float *tgt, const float *w, long V, float inv_count,
                         void *g, double *loss, void *stream)
{
  if (!yhead || !tgt || !w || !g || !loss || N < 1) return qesb_fail(QESB_ERR_ARG, "qesb_net_mse: bad arguments");
  k_mse<<<gs_blocks(V), 256, 0, (cudaStream_t)stream>>>(yhead, N, tgt, w, V, inv_count, (__nv_bfloat16 *)g, loss);
  NET_CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_net_mse_coarse(const float *yhead, int N, const float *tgt, const float *w, int D, int H, int W,
                                int F, float beta, void *g, double *loss, void *stream)
{
  if (!yhead || !tgt || !w || !g || !loss || F < 1 || D % F || H % F || W % F)
    return qesb_fail(QESB_ERR_ARG, "qesb_net_mse_coarse: bad arguments");
  const long nc = (long)(D / F) * (H / F) * (W / F);
  k_mse_coarse<<<gs_blocks(nc, 128), 128, 0, (cudaStream_t)stream>>>(yhead, N, tgt, w, D, H, W, F, beta,
                                                                       (__nv_bfloat16 *)g, loss);
  NET_CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_net_adam_conv(float *Wt, float *m, float *v, const float *dW, int cin, int cout, int cout_real,
                               void *Bm, int Kp, void *Bd, int Kd, float lr, float b1, float b2, float eps,
                               int step, float grad_scale, void *stream)
{
  if (!Wt || !m || !v || !dW || !Bm || step < 1) return qesb_fail(QESB_ERR_ARG, "qesb_net_adam_conv: bad arguments");
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  const long n = 27L * cin * cout;
  k_adam_conv<<<gs_blocks(n), 256, 0, (cudaStream_t)stream>>>(Wt, m, v, dW, cin, cout, cout_real,
                                                              (__nv_bfloat16 *)Bm, Kp, (__nv_bfloat16 *)Bd, Kd, lr,
                                                              b1, b2, eps, c1, c2, grad_scale);
  NET_CK(cudaGetLastError());
  return QESB_OK;
}

qesb_status qesb_net_adam_vec(float *p, float *m, float *v, const float *g, int n, float lr, float b1, float b2,
                              float eps, int step, float grad_scale, void *stream)
{
  if (!p || !m || !v || !g || n <= 0 || step < 1) return qesb_fail(QESB_ERR_ARG, "qesb_net_adam_vec: bad arguments");
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_adam_vec<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(p, m, v, g, n, lr, b1, b2, eps, c1, c2, grad_scale);
  NET_CK(cudaGetLastError());
  return QESB_OK;
}

}  // extern "C"
