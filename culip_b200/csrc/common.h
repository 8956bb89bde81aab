// Shared host-side definitions for the culipx library: status handling and
// the C-ABI export macro.  Includes the public C header.
#pragma once

#include "culipx.h"

#include <cstdio>
#include <string>

#define CULIPX_API __attribute__((visibility("default")))

namespace culipx {

// Records a message for culipx_last_error() (thread-local) and returns `status`.
int fail(int status, const char* fmt, ...);
void clear_error();

}  // namespace culipx
