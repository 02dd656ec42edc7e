// Device-side types and helpers shared by the solver kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace qesb {

constexpr float kOmega = 1.78f;  // over-relaxation factor, src/winds/Solver.h:83
constexpr int kGX = 8;           // x guard cells on each side of the padded layout
constexpr int kGY = 8;           // y guard rows on each side
constexpr int kMaxTileRows = 64; // tallest tiled-kernel tile (rows incl. halo)

// Grid sizes in cells (X, Y, Z = nx-1, ny-1, nz-1), in faces (FX, FY, FZ =
// nx, ny, nz) and the padded cell layout (PX, PY, PLANE).
struct DevGrid {
  int X, Y, Z;
  int FX, FY, FZ;
  long XY, FXY;
  int PX, PY;
  long PLANE;
  __host__ __device__ long cell(int i, int j, int k) const { return i + (long)j * X + (long)k * XY; }
  __host__ __device__ long face(int i, int j, int k) const { return i + (long)j * FX + (long)k * FXY; }
  __host__ __device__ long pad(int i, int j, int k) const
  {
    return (long)k * PLANE + (long)(j + kGY) * PX + (i + kGX);
  }
};

// Device-side state of one solve; polled by the kernels so the iteration
// loop needs no host round trip per iteration.
struct SolveState {
  int done;       // 1 once the loop condition has failed
  int it;         // iterations completed
  int converged;  // stop came from max|dlambda| <= tol
  int nan;        // a NaN error was met
  double residual;
  int cur;        // lambda buffer (0 or 1) written by the last launch that ran
  int redo;       // >0: the converging launch ran past the stop; re-run this many iterations
  int redo_t0;    // first iteration of that launch
  int redo_par;   // its output buffer
  unsigned blocks_done;  // CTAs of the current black half-sweep that have finished
  unsigned long long t_done;  // %globaltimer (ns) when a batched solve's loop ended
  double wacc;    // window rule: max|lambda - snapshot| being gathered by the current check
  double wdrift;  // window rule: the last completed window's max|lambda - snapshot|
};

__device__ __forceinline__ unsigned long long global_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool is_solid(int flag) { return flag == 0 || flag == 2; }

__device__ __forceinline__ float warp_max_f(float v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_max_d(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = (w > v || w != w) ? w : v;  // NaN propagates
  }
  return v;
}

// Non-negative doubles (and NaN, whose bits exceed every finite value's)
// order like their 64-bit patterns, so atomicMax on the bits is a max.
__device__ __forceinline__ void atomic_max_nonneg(double *p, double v)
{
  atomicMax(reinterpret_cast<unsigned long long *>(p), (unsigned long long)__double_as_longlong(v));
}

// Block-wide max of a non-negative double into *dst, one atomic per block.
// Every thread of the block must call it.
__device__ __forceinline__ void block_max_to(double *dst, double v)
{
  __shared__ double s_part[32];
  v = warp_max_d(v);
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int lane = tid & 31, wid = tid >> 5;
  if (lane == 0) s_part[wid] = v;
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
    double x = lane < nw ? s_part[lane] : 0.0;
    x = warp_max_d(x);
    if (lane == 0 && x != 0.0) atomic_max_nonneg(dst, x);
  }
}

}  // namespace qesb
