/* Drop-in for formats/formats.h (reference formats/formats.h:1-102):
 * matrix_shape, coo_matrix, csr_matrix<T> (pad, spmv_bytes), slell_params
 * and slell_matrix<E, memory_space> with the reference's members and layout
 * (the sliced-ELL arrays are bit-identical to the reference's conversion).
 *
 * Beyond the reference: slell_matrix also records its shortest and tallest
 * slice (min_slice_height, max_slice_height; equal to slice_height unless
 * var_height), which the variable-height launch checks need, and
 * spmv_bytes counts vec_elt_size bytes per vector entry (the reference
 * counts sizeof(int) whatever the argument, formats.h:77). */
#ifndef MATRIX_FORMATS_H
#define MATRIX_FORMATS_H

#include <stddef.h>

#include "util/cuda/vector.h"

struct matrix_shape {
  int n_rows, n_cols, n_nz;
};

template <class T> struct coo_matrix : matrix_shape {
  vector<int> rows, cols;
  vector<T> elms;
};

template <class T> struct csr_matrix : matrix_shape {
  vector<int, host_memory_space_tag> row_ptr, cols;
  vector<T, host_memory_space_tag> elms;
  /* append empty rows up to a multiple of k (k a power of two) */
  void pad(int k)
  {
    k--;
    const int n_padded_rows = (n_rows + k) & ~k;
    const int last = row_ptr.back();
    for (; n_rows < n_padded_rows; n_rows++)
      row_ptr.push_back(last);
  }

  unsigned spmv_bytes() const
  {
    return (unsigned)(sizeof(unsigned) * (row_ptr.size() + cols.size()) +
                      sizeof(T) * (elms.size() + 2 * (size_t)n_rows));
  }
};

struct slell_params {
  unsigned S, H, V, D;
};

template <typename E, typename memory_space> struct slell_matrix : matrix_shape {
  vector<unsigned, memory_space> slice_ptr;
  vector<unsigned, memory_space> cols;
  vector<E, memory_space> elms;
  unsigned slice_height;
  unsigned n_slices;
  unsigned hblock;
  bool var_height;
  bool diags;
  unsigned min_slice_height, max_slice_height;

  slell_matrix(const slell_matrix<E, host_memory_space_tag> &m)
      : matrix_shape(m), slice_ptr(m.slice_ptr), cols(m.cols), elms(m.elms),
        slice_height(m.slice_height), n_slices(m.n_slices), hblock(m.hblock),
        var_height(m.var_height), diags(m.diags), min_slice_height(m.min_slice_height),
        max_slice_height(m.max_slice_height)
  {
  }

  slell_matrix(const matrix_shape &m)
      : matrix_shape(m), slice_height(0), n_slices(0), hblock(1), var_height(false),
        diags(false), min_slice_height(0), max_slice_height(0)
  {
  }

  slell_matrix()
      : slice_height(0), n_slices(0), hblock(1), var_height(false), diags(false),
        min_slice_height(0), max_slice_height(0)
  {
    n_rows = n_cols = n_nz = 0;
  }

  unsigned spmv_bytes(bool effective = false, int vec_elt_size = sizeof(E))
  {
    return (unsigned)(sizeof(unsigned) * slice_ptr.size() +
                      sizeof(unsigned) * (effective ? (size_t)n_nz : cols.size()) +
                      sizeof(E) * (effective ? (size_t)n_nz : elms.size()) +
                      (size_t)vec_elt_size * 2 * (size_t)n_rows);
  }

  /* First element of the slice starting at `row` (host matrices), or NULL
   * when no slice starts there (formats.h:80-101). */
  E *slice_elt_ptr(unsigned row, unsigned &slice_hint)
  {
    const int slice_ents = (int)(slice_ptr.size() / (n_slices + 1));
    unsigned slice;
    if (!var_height) {
      slice = row / slice_height;
      if (row % slice_height)
        return NULL;
    } else {
      for (slice = slice_hint; slice <= n_slices && slice_ptr[slice * slice_ents + 1] != row;
           slice++) {
      }
      if (slice > n_slices)
        return NULL;
      slice_hint = slice;
    }
    return &elms[slice_ptr[slice * slice_ents]];
  }
};

#endif
