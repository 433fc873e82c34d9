/* Drop-in for util/cuda/initialize.h (reference util/cuda/initialize.h:1-12,
 * util/cuda/initialize.cu:17-42): ispm_initialize() checks that the current
 * device is sm_100 and sets cudaDeviceMapHost, aborting on a mismatch as the
 * reference does; get_device_string() names the current device as
 * "dddd:bb:dd (name)". */
#ifndef ISPM_INITIALIZE_H
#define ISPM_INITIALIZE_H

#include "ispm_compat_detail.h"

inline void ispm_initialize() { ispm_compat::check(ispm_c::ispm_initialize(), "ispm_initialize"); }

struct DeviceIDString {
  char str[32];
};

inline DeviceIDString get_device_string()
{
  DeviceIDString s;
  ispm_compat::check(ispm_c::ispm_get_device_string(s.str, (int)sizeof(s.str)),
                     "get_device_string");
  return s;
}

#endif
