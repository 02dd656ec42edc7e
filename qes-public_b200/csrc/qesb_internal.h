// Internal helpers shared by the library's translation units.
#pragma once
#include "qesb.h"

// Records a thread-local message for qesb_last_error() and returns `s`.
qesb_status qesb_fail(qesb_status s, const char *fmt, ...);

// Returns from the calling function when `x` is not QESB_OK.
#define CKS_FWD(x)                    \
  do {                                \
    const qesb_status s_ = (x);       \
    if (s_ != QESB_OK) return s_;     \
  } while (0)

// The handle's base grid counts and device (for the library's other parts).
qesb_status qesb_handle_grid(qesb_handle *h, int *Nx, int *Ny, int *Nz, int *device);

// Wall::defineWalls + Wall::solverCoefficients (stair-step walls) on the
// device: e..n (cell arrays) from a flag field already on the device, on the
// given stream; dz on the device (nz - 1 values, as the grid's dz_array).
qesb_status qesb_city_walls_dev(int Nx, int Ny, int Nz, float dx, const float *d_dz, const int *d_flag, float *e,
                                float *f, float *g, float *hc, float *m, float *n, void *stream);

// Forward convolution of one input whose output channel 0 alone is stored:
// y0 FP32 [V] (the network's head; arguments as qesb_conv3d_items).
qesb_status qesb_conv3d_head(const void *x1, int c1, int items, int D, int H, int W, const void *Bm, int Kp, int N,
                             float *y0, const float *bias, int relu, int *err, void *stream);

// A small transfer run as a kernel on `stream` (no copy engine): dst and src
// device memory or the device alias of mapped pinned host memory, bytes a
// multiple of 4. The caller waits for the stream before reading dst.
qesb_status qesb_copy_small(void *dst, const void *src, size_t bytes, void *stream);
