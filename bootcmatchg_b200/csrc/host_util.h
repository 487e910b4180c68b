// Host-side helpers shared by the library's C++ translation units: the
// thread-local error message behind bcmg_last_error() and a status macro.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <string>

#include "bcmg.h"

namespace bcmg {

// Records a formatted message as this thread's last error and returns code.
bcmg_status set_error(bcmg_status code, const char *fmt, ...);
void clear_error();

}  // namespace bcmg

#define BCMG_TRY(expr)                          \
  do {                                          \
    bcmg_status _st = (expr);                   \
    if (_st != BCMG_OK) return _st;             \
  } while (0)
