/* Shared plumbing of the C++ drop-in headers (include/compat/...).
 *
 * The drop-in headers give a caller of the reference library the reference's
 * own include paths, types and template signatures (formats/formats.h,
 * formats/conversion.h, plan/plan.h, cuda/spmv/kernel-iface.h,
 * util/cuda/sblas.h, util/cuda/vector.h, fastainv/fastainv.h,
 * fastainv/droptol-tuning.h, util/cuda/initialize.h), implemented inline over
 * the C ABI of libispm_b200.so.  Build a caller with
 *     -I<repo>/include/compat  -L<repo>/ispm-sparse-lib_b200 -lispm_b200 -lcudart
 * in place of the reference's include directory and libispm0-pic.a.
 *
 * The C ABI is declared inside namespace ispm_c so that its names cannot
 * collide with the reference's C++ names (the reference's C++
 * `void ispm_initialize()` and the C ABI's `int ispm_initialize(void)`).  A
 * translation unit that uses these headers must not include ispm_b200.h
 * before them.
 *
 * Error behaviour follows the reference: a failing CUDA or library call
 * prints the cause and aborts (util/cuda/check.h:8-15), and an SpMV launch
 * with unsupported parameters launches nothing (cuda/spmv/dispatch.h). */
#ifndef ISPM_COMPAT_DETAIL_H
#define ISPM_COMPAT_DETAIL_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#ifdef ISPM_B200_H
#error "include the drop-in headers before ispm_b200.h (or without it)"
#endif

namespace ispm_c {
#include "../ispm_b200.h"
}

namespace ispm_compat {

template <class T> struct dtype_of;
template <> struct dtype_of<float> {
  static const int value = ISPM_F32;
};
template <> struct dtype_of<double> {
  static const int value = ISPM_F64;
};

/* Abort with the library's message unless status is ISPM_OK. */
inline void check(int status, const char *what)
{
  if (status != ISPM_OK) {
    fprintf(stderr, "ispm: %s failed: %s (%s)\n", what, ispm_c::ispm_error_string(status),
            ispm_c::ispm_last_error());
    abort();
  }
}

}  // namespace ispm_compat

#endif
