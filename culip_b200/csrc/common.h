// Shared host-side definitions for the culipx library: status handling and
// the C-ABI export macro.  Includes the public C header.
#pragma once

#include "culipx.h"

#include <cstdio>
#include <string>

#define CULIPX_API __attribute__((visibility("default")))

namespace culipx {

// An FP32 factor inverts a 2x2 pivot in FP64 when it is ill-conditioned:
// |d11 d22 - d12^2| < bound (|d11 d22| + d12^2).  The ratio is 1 for a
// diagonal pivot and 0 for a singular one; its error in single precision is
// about 6e-8 / ratio, so below bound = 1e-3 the Givens solve of FP32 would
// lose more than four of its seven digits.  Bunch-Kaufman and rook pivoting
// only accept 2x2 pivots with |d11 d22| < alpha^2 d12^2 (alpha = 0.64), i.e.
// a ratio above (1 - alpha^2) / (1 + alpha^2) = 0.42, so the FP64 branch is
// taken by given (static) pivots.  0 turns it off (the reference's FP32
// arithmetic throughout).
constexpr double kPivotFp64Default = 1e-3;

// Records a message for culipx_last_error() (thread-local) and returns `status`.
int fail(int status, const char* fmt, ...);
void clear_error();

}  // namespace culipx
