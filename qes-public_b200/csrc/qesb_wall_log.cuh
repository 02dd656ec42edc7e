// Log-law wall treatment of the stair-step walls after a solve: the second
// part of Wall::wallLogBC (src/winds/Wall.cpp:656-803) on the walls that
// Wall::defineWalls lists (src/winds/Wall.cpp:287-340), as qesWindsMain.cpp:
// 157-166 applies it when logLawFlag = 1 (u0 <- u, wallLogBC, u <- u0), here in
// place on the solved winds.
//
// Each fluid cell (flag not 0 or 2) next to a solid one (flag 0 or 2) gets a
// bit per side: below, above, back (i > 0), front, right (j > 0), left, the
// neighbours taken by flat cell index exactly as Domain::cellAdd gives them
// (the front and left neighbours of the last column and row run on to the next
// row and plane); cells flagged 8 are not listed. The six sides are then
// treated in the reference's order, one launch each. Within one side no cell
// reads a face another cell of that side writes (the neighbour read is the
// cell's fluid side), so each launch is fully parallel; across sides the order
// matters (a face may sit in several lists, and a later side reads what an
// earlier one wrote), and the launches keep it.
//
// Per wall face: with (a, b) the two wall-parallel components of the
// neighbour face one cell into the fluid, wind_dir = atan2(b, a), |U| =
// sqrt(a^2 + b^2) (in double, as the reference's pow(x, 2.0) evaluates it);
// 20 steps of u* <- vk (|U| - u*/vk log(d2/d1)) / log(d1/z0) from u* = 0.1;
// then the normal component is zeroed and the parallel ones set to
// vel_mag1 (cos, sin)(wind_dir). The two logarithms are constants of the side
// and come from the host's logf, the function the reference calls; atan2, cos
// and sin are evaluated in double and rounded to float.
#pragma once
#include "qesb_device.cuh"

namespace qesb {

enum WallSide { kWallBelow = 0, kWallAbove, kWallBack, kWallFront, kWallRight, kWallLeft };

__device__ __forceinline__ bool wall_solid(int f) { return f == 0 || f == 2; }

// bits[c] for cells k in [1, Z - 2] (all i, j); *cut = 1 if one of those cells
// carries a cut-cell flag (7 or 8), whose walls this treatment does not cover.
__global__ void k_wall_bits(DevGrid G, const int *__restrict__ flag, uint8_t *__restrict__ bits, int *cut)
{
  const int j = blockIdx.y, k = blockIdx.z + 1;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x) {
    const long c = G.cell(i, j, k);
    const int f = flag[c];
    if (f == 7 || f == 8) atomicOr(cut, 1);
    unsigned b = 0;
    if (!wall_solid(f) && f != 8) {
      if (wall_solid(flag[c - G.XY])) b |= 1u << kWallBelow;
      if (wall_solid(flag[c + G.XY])) b |= 1u << kWallAbove;
      if (i > 0 && wall_solid(flag[c - 1])) b |= 1u << kWallBack;
      if (wall_solid(flag[c + 1])) b |= 1u << kWallFront;
      if (j > 0 && wall_solid(flag[c - G.X])) b |= 1u << kWallRight;
      if (wall_solid(flag[c + G.X])) b |= 1u << kWallLeft;
    }
    bits[c] = (uint8_t)b;
  }
}

// One side. a, b: the wall-parallel components (wind_dir = atan2(b, a)); nrm:
// the normal one. l21 = logf(d2 / d1), l10 = logf(d1 / z0).
template <int SIDE>
__global__ void k_wall_log(DevGrid G, const uint8_t *__restrict__ bits, const int *cut, float *u, float *v, float *w,
                           float l21, float l10)
{
  if (*cut) return;
  const int j = blockIdx.y, k = blockIdx.z + 1;
  float *a = (SIDE == kWallBack || SIDE == kWallFront) ? v : u;
  float *b = (SIDE == kWallBelow || SIDE == kWallAbove) ? v : w;
  float *nrm = (SIDE == kWallBelow || SIDE == kWallAbove) ? w : (SIDE == kWallBack || SIDE == kWallFront) ? u : v;
  const long step = (SIDE == kWallBelow || SIDE == kWallAbove) ? G.FXY : (SIDE == kWallBack || SIDE == kWallFront) ? 1 : G.FX;
  const long dnb = (SIDE == kWallBelow || SIDE == kWallBack || SIDE == kWallRight) ? step : -step;
  const float vk = 0.4f;
  for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < G.X; i += gridDim.x * blockDim.x) {
    if (!(bits[G.cell(i, j, k)] & (1u << SIDE))) continue;
    const long f = G.face(i, j, k), nb = f + dnb;
    const float av = a[nb], bv = b[nb];
    const float wind_dir = (float)atan2((double)bv, (double)av);
    const float mag2 = (float)sqrt((double)av * (double)av + (double)bv * (double)bv);
    float ustar = 0.1f, mag1 = 0.0f;
#pragma unroll 1
    for (int it = 0; it < 20; ++it) {
      mag1 = mag2 - (ustar / vk) * l21;
      ustar = vk * mag1 / l10;
    }
    nrm[f] = 0.0f;
    a[f] = mag1 * (float)cos((double)wind_dir);
    b[f] = mag1 * (float)sin((double)wind_dir);
  }
}

}  // namespace qesb
