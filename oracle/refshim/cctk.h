// Test infrastructure only: a minimal stand-in for the Cactus flesh header
// so that the reference hot-path sources compile unmodified on the host CPU.
// Nothing in the product library includes this file.
#ifndef AXREF_SHIM_CCTK_H
#define AXREF_SHIM_CCTK_H

#include <cassert>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <strings.h>

typedef double CCTK_REAL;
typedef int CCTK_INT;
typedef int CCTK_BOOLEAN;

#define CCTK_DEVICE
#define CCTK_HOST
#define CCTK_ATTRIBUTE_ALWAYS_INLINE
#define ARITH_INLINE
#define ARITH_DEVICE
#define ARITH_HOST

// Cactus keyword parameters compare case-insensitively.
#define CCTK_EQUALS(a, b) (strcasecmp((a), (b)) == 0)

[[noreturn]] void axref_fatal(const char *msg);
#define CCTK_ERROR(msg) axref_fatal(msg)
#define CCTK_VERROR(...)                                                       \
  do {                                                                         \
    char axref_buf_[512];                                                      \
    snprintf(axref_buf_, sizeof axref_buf_, __VA_ARGS__);                      \
    axref_fatal(axref_buf_);                                                   \
  } while (0)
#define CCTK_VINFO(...)                                                        \
  do {                                                                         \
  } while (0)
#define CCTK_INFO(msg)                                                         \
  do {                                                                         \
  } while (0)
#define CCTK_WARN(lvl, msg)                                                    \
  do {                                                                         \
  } while (0)

#endif
