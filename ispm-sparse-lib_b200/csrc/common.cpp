// Error reporting and host threading shared by the whole library.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <thread>

#include "ispm_internal.h"

namespace ispm {

static thread_local std::string g_last_error;

int fail(int status, const char *fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

void clear_error() { g_last_error.clear(); }

int host_threads()
{
  static int n = [] {
    const char *e = getenv("ISPM_NUM_THREADS");
    int v = e ? atoi(e) : 0;
    if (v <= 0)
      v = (int)std::thread::hardware_concurrency();
    return v > 0 ? v : 1;
  }();
  return n;
}

}  // namespace ispm

extern "C" {

const char *ispm_error_string(int status)
{
  switch (status) {
  case ISPM_OK: return "ok";
  case ISPM_ERR_INVALID: return "invalid argument";
  case ISPM_ERR_CUDA: return "CUDA error";
  case ISPM_ERR_NOMEM: return "out of memory";
  case ISPM_ERR_ARCH: return "unsupported device architecture";
  case ISPM_ERR_BREAKDOWN: return "solver breakdown";
  case ISPM_ERR_NOT_CONVERGED: return "not converged";
  case ISPM_ERR_TIMEOUT: return "device wait timed out";
  case ISPM_ERR_TOO_LARGE: return "size above supported maximum";
  default: return "unknown status";
  }
}

const char *ispm_last_error(void) { return ispm::g_last_error.c_str(); }

const char *ispm_version(void) { return "ispm-b200 0.1 (sm_100a)"; }

}  // extern "C"
