/* Drop-in for util/cuda/devmem.h (reference util/cuda/devmem.h:1-25):
 * devmem<T> marks a T that lives in device memory, so device and host
 * pointers are distinct types; uncast_devmem gives the plain pointer. */
#ifndef DEVMEM_H
#define DEVMEM_H

template <class T> class devmem {
  unsigned char bytes_[sizeof(T)];
};

template <typename T> static inline T *uncast_devmem(devmem<T> *p)
{
  return reinterpret_cast<T *>(p);
}

template <typename T> static inline const T *uncast_devmem(const devmem<T> *p)
{
  return reinterpret_cast<const T *>(p);
}

#endif
