// Learned warm start: tensor-core kernels (tcgen05, BF16 operands, FP32
// accumulation in TMEM) for the 3D-convolution network, and their C ABI.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "qesb.h"
#include "qesb_internal.h"
#include "qesb_umma.cuh"

using namespace qesb;

namespace {

constexpr uint32_t kWaitLimit = 1u << 26;  // mbarrier polls before a kernel gives up

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
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
  if (warp == 0) umma::tmem_alloc(&tmem_base, ncols);
  if (tid == 0) {
    umma::mbar_init(&mbar, 1);
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
