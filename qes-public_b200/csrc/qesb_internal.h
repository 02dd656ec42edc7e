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
