// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into, or called by, the
// product library.  Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg load the shared object built from this file.
//
// extern "C" wrappers around the reference's own host code, compiled IN PLACE
// from the reference source tree (see oracle/Makefile; nothing is copied):
//   formats/conversion.h:338-414  csr_to_slell
//   formats/conversion.h:416-492  csr_to_slell_guess_format
//   fastainv/fastainv.cpp:395-566 fastainv_sym (compiled from its own .cpp)
//   fastainv/droptol-tuning.h:4-103 DroptolTuner
// The wrappers only marshal plain arrays into the reference's containers and
// back out; every computed value comes from the reference's code.

#include <climits>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <algorithm>
#include <vector>

#include "formats/formats.h"
#include "formats/conversion.h"
#include "fastainv/fastainv.h"
#include "fastainv/droptol-tuning.h"

extern "C" {

struct ref_slell {
  int n_rows, n_cols, n_nz;
  unsigned slice_height, n_slices, hblock;
  int var_height, diags;
  long long n_slice_ptr, n_cols_arr, n_elms;
  unsigned *slice_ptr;
  unsigned *cols;
  void *elms;
};

struct ref_csr {
  int n_rows, n_cols, n_nz;
  int *row_ptr;
  int *cols;
  void *elms;
};

}

// The reference's csr_to_slell_guess_format reads row_ptr entries past n_rows
// for small matrices (conversion.h:429,438 examine rows_to_examine rounded up
// to 32 before the CSR is padded).  We give it a row_ptr that already carries
// enough trailing copies of row_ptr[n] so those reads are defined and equal
// to "empty rows" -- the same meaning the padded matrix gives them.
enum { EXTRA_ROW_PTR = 1024 };

template <class T>
static void fill_csr(csr_matrix<T> &A, int n_rows, int n_cols, const int *row_ptr,
                     const int *cols, const T *elms)
{
  A.n_rows = n_rows;
  A.n_cols = n_cols;
  A.n_nz = row_ptr[n_rows];
  A.row_ptr.assign(row_ptr, row_ptr + n_rows + 1);
  A.cols.assign(cols, cols + row_ptr[n_rows]);
  A.elms.assign(elms, elms + row_ptr[n_rows]);
}

template <class T>
static void export_slell(const slell_matrix<T, host_memory_space_tag> &B, ref_slell *out)
{
  out->n_rows = B.n_rows;
  out->n_cols = B.n_cols;
  out->n_nz = B.n_nz;
  out->slice_height = B.slice_height;
  out->n_slices = B.n_slices;
  out->hblock = B.hblock;
  out->var_height = B.var_height;
  out->diags = B.diags;
  out->n_slice_ptr = B.slice_ptr.size();
  out->n_cols_arr = B.cols.size();
  out->n_elms = B.elms.size();
  out->slice_ptr = (unsigned *)malloc(sizeof(unsigned) * (B.slice_ptr.size() + 1));
  out->cols = (unsigned *)malloc(sizeof(unsigned) * (B.cols.size() + 1));
  out->elms = malloc(sizeof(T) * (B.elms.size() + 1));
  if (!B.slice_ptr.empty())
    memcpy(out->slice_ptr, &B.slice_ptr[0], sizeof(unsigned) * B.slice_ptr.size());
  if (!B.cols.empty())
    memcpy(out->cols, &B.cols[0], sizeof(unsigned) * B.cols.size());
  if (!B.elms.empty())
    memcpy(out->elms, &B.elms[0], sizeof(T) * B.elms.size());
}

template <class T>
static int conv(int guess, int n_rows, int n_cols, const int *row_ptr, const int *cols,
                const T *elms, int S, int hblock, int var_height, int use_diags,
                int examine_ratio, int min_height, ref_slell *out, int *padded_rows)
{
  csr_matrix<T> A;
  fill_csr(A, n_rows, n_cols, row_ptr, cols, elms);
  for (int i = 0; i < EXTRA_ROW_PTR; i++)
    A.row_ptr.push_back(row_ptr[n_rows]);
  slell_matrix<T, host_memory_space_tag> B =
      guess ? csr_to_slell_guess_format(A, examine_ratio, min_height)
            : csr_to_slell(A, S, hblock, var_height != 0, use_diags != 0, min_height);
  export_slell(B, out);
  if (padded_rows)
    *padded_rows = A.n_rows;   // csr_to_slell pads the caller's CSR in place
  return 0;
}

extern "C" {

int ref_csr_to_slell(int f64, int n_rows, int n_cols, const int *row_ptr, const int *cols,
                     const void *elms, int S, int hblock, int var_height, int use_diags,
                     int min_height, ref_slell *out, int *padded_rows)
{
  if (f64)
    return conv<double>(0, n_rows, n_cols, row_ptr, cols, (const double *)elms, S, hblock,
                        var_height, use_diags, 1, min_height, out, padded_rows);
  return conv<float>(0, n_rows, n_cols, row_ptr, cols, (const float *)elms, S, hblock,
                     var_height, use_diags, 1, min_height, out, padded_rows);
}

int ref_csr_to_slell_guess_format(int f64, int n_rows, int n_cols, const int *row_ptr,
                                  const int *cols, const void *elms, int examine_ratio,
                                  int min_height, ref_slell *out, int *padded_rows)
{
  if (f64)
    return conv<double>(1, n_rows, n_cols, row_ptr, cols, (const double *)elms, 0, 0, 0, 0,
                        examine_ratio, min_height, out, padded_rows);
  return conv<float>(1, n_rows, n_cols, row_ptr, cols, (const float *)elms, 0, 0, 0, 0,
                     examine_ratio, min_height, out, padded_rows);
}

void ref_slell_free(ref_slell *m)
{
  free(m->slice_ptr);
  free(m->cols);
  free(m->elms);
  m->slice_ptr = 0;
  m->cols = 0;
  m->elms = 0;
}

static void count_progress(void *v)
{
  if (v)
    ++*(long long *)v;
}

}  // extern "C"

template <class O>
static void export_csr(const csr_matrix<O> &A, ref_csr *out)
{
  out->n_rows = A.n_rows;
  out->n_cols = A.n_cols;
  out->n_nz = A.n_nz;
  size_t nnz = A.cols.size();
  out->row_ptr = (int *)malloc(sizeof(int) * (A.row_ptr.size() + 1));
  out->cols = (int *)malloc(sizeof(int) * (nnz + 1));
  out->elms = malloc(sizeof(O) * (nnz + 1));
  memcpy(out->row_ptr, &A.row_ptr[0], sizeof(int) * A.row_ptr.size());
  if (nnz) {
    memcpy(out->cols, &A.cols[0], sizeof(int) * nnz);
    memcpy(out->elms, &A.elms[0], sizeof(O) * nnz);
  }
}

extern "C" {

// out_f64: 1 -> fastainv_sym<double,double>, 0 -> fastainv_sym<double,float>
int ref_fastainv_sym(int out_f64, int n, const int *row_ptr, const int *cols,
                     const double *elms, long long max_elts, double droptol,
                     ref_csr *ainv1, ref_csr *ainv2, long long *progress_calls)
{
  csr_matrix<double> A;
  fill_csr(A, n, n, row_ptr, cols, elms);
  long long calls = 0;
  bool ok;
  if (out_f64) {
    csr_matrix<double> G1, G2;
    ok = fastainv_sym(G1, G2, A, count_progress, &calls, max_elts, droptol);
    if (ok) {
      export_csr(G1, ainv1);
      export_csr(G2, ainv2);
    }
  } else {
    csr_matrix<float> G1, G2;
    ok = fastainv_sym(G1, G2, A, count_progress, &calls, max_elts, droptol);
    if (ok) {
      export_csr(G1, ainv1);
      export_csr(G2, ainv2);
    }
  }
  if (progress_calls)
    *progress_calls = calls;
  return ok ? 1 : 0;
}

void ref_csr_free(ref_csr *m)
{
  free(m->row_ptr);
  free(m->cols);
  free(m->elms);
  m->row_ptr = 0;
  m->cols = 0;
  m->elms = 0;
}

void *ref_tuner_new(double lo, double hi) { return new DroptolTuner(lo, hi); }
void ref_tuner_free(void *t) { delete (DroptolTuner *)t; }
double ref_tuner_get_droptol(void *t) { return ((DroptolTuner *)t)->getDroptol(); }
double ref_tuner_get_best_droptol(void *t) { return ((DroptolTuner *)t)->getBestDroptol(); }
void ref_tuner_note_time(void *t, double time) { ((DroptolTuner *)t)->noteTime(time); }
void ref_tuner_restart(void *t) { ((DroptolTuner *)t)->restart(); }
void ref_tuner_reset_phase(void *t) { ((DroptolTuner *)t)->resetPhase(); }
int ref_tuner_iterations(void *t) { return ((DroptolTuner *)t)->iterations(); }

}
