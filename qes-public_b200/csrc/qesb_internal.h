// Internal helpers shared by the library's translation units.
#pragma once
#include "qesb.h"

// Records a thread-local message for qesb_last_error() and returns `s`.
qesb_status qesb_fail(qesb_status s, const char *fmt, ...);
