/* Drop-in for util/cuda/vector.h (reference util/cuda/vector.h:1-95):
 * vector<T, host_memory_space_tag> is a std::vector<T> that can be built
 * from or assigned a device vector; vector<T, device_memory_space_tag> owns
 * zero-filled device memory (cudaMalloc) and hands out devmem<T> pointers.
 *
 * Beyond the reference: a device vector can be copied (device-to-device),
 * assigned a host vector (host-to-device copy; the reference's
 * spmv_plan::update_device_matrix_coefs relies on that assignment), and
 * resize() keeps the old contents (zero-filling the new tail). */
#ifndef VECTOR_H
#define VECTOR_H

#include <cuda_runtime.h>

#include <vector>

#include "check.h"
#include "cudamemcpy.h"
#include "devmem.h"

struct host_memory_space_tag {};
struct device_memory_space_tag {};

template <typename T, typename memory_space = host_memory_space_tag> class vector;

template <typename T> class vector<T, device_memory_space_tag>;

template <typename T> class vector<T, host_memory_space_tag> : public std::vector<T> {
  typedef std::vector<T> parent;

 public:
  vector() {}
  vector(size_t n) : parent(n) {}
  vector(size_t n, T v) : parent(n, v) {}
  vector(const vector<T, device_memory_space_tag> &v);
  vector<T, host_memory_space_tag> &operator=(const vector<T, device_memory_space_tag> &v);
};

template <typename T> class vector<T, device_memory_space_tag> {
  devmem<T> *p_;
  size_t n_;

  static devmem<T> *alloc(size_t n)
  {
    if (!n)
      return nullptr;
    void *p = nullptr;
    CUDA_CHECK(cudaMalloc(&p, n * sizeof(T)));
    CUDA_CHECK(cudaMemset(p, 0, n * sizeof(T)));
    return static_cast<devmem<T> *>(p);
  }

 public:
  vector() : p_(nullptr), n_(0) {}
  vector(size_t n) : p_(alloc(n)), n_(n) {}
  vector(const vector<T, host_memory_space_tag> &v) : p_(alloc(v.size())), n_(v.size())
  {
    copy(p_, v.data(), n_);
  }
  vector(const vector &v) : p_(alloc(v.n_)), n_(v.n_) { copy(p_, v.p_, n_); }
  template <typename TI> vector(const TI first, const TI last) : p_(nullptr), n_(0)
  {
    assign(first, last);
  }
  ~vector()
  {
    if (p_)
      cudaFree(p_);
  }
  vector &operator=(const vector &v)
  {
    if (this != &v) {
      if (n_ != v.n_) {
        vector t(v.n_);
        swap(t);
      }
      copy(p_, v.p_, n_);
    }
    return *this;
  }
  vector &operator=(const vector<T, host_memory_space_tag> &v)
  {
    if (n_ != v.size()) {
      vector t(v.size());
      swap(t);
    }
    copy(p_, v.data(), n_);
    return *this;
  }
  void swap(vector &o)
  {
    devmem<T> *p = p_;
    size_t n = n_;
    p_ = o.p_;
    n_ = o.n_;
    o.p_ = p;
    o.n_ = n;
  }
  template <typename TI> void assign(const TI first, const TI last)
  {
    if (first + size() < last)
      resize(last - first);
    copy(p_, &*first, last - first);
  }
  template <typename TI> void assign_async(const TI first, const TI last)
  {
    if (first + size() < last)
      resize(last - first);
    copy_async(p_, &*first, last - first);
  }
  void resize(size_t n)
  {
    if (n == n_)
      return;
    vector t(n);
    copy(t.p_, p_, n < n_ ? n : n_);
    swap(t);
  }
  devmem<T> *data() { return p_; }
  const devmem<T> *data() const { return p_; }
  T *udata() { return uncast_devmem(p_); }
  size_t size() const { return n_; }
};

template <typename T>
vector<T, host_memory_space_tag>::vector(const vector<T, device_memory_space_tag> &v)
    : parent(v.size())
{
  copy(this->data(), v.data(), v.size());
}

template <typename T>
vector<T, host_memory_space_tag> &
vector<T, host_memory_space_tag>::operator=(const vector<T, device_memory_space_tag> &v)
{
  if (this->size() < v.size())
    this->resize(v.size());
  copy(this->data(), v.data(), v.size());
  return *this;
}

#endif
