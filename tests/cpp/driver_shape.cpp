// A caller in the shape of the reference's external user (the foam-extend
// ispmCudaSolvers driver, reference README.md:5-9), written only against the
// reference's headers and template signatures.  It builds against the
// reference's own headers (host part) and against this library's drop-in
// headers (include/compat, host and device parts) without a change.
//
// Host part: CSR -> sliced-ELL in three shapes, the format guess, the
// approximate inverse in double and float, and a drop-tolerance search.  It
// prints one line per result: sizes and an FNV-1a hash of every array, so
// two builds can be compared bit for bit.
// Device part (DRIVER_DEVICE): device upload, both launch_spmv_kernel
// overloads for (double, double) and (double, float), a launch with
// unsupported parameters (must launch nothing), the sblas calls, and the
// DEFAULT and EXHAUSTIVE plans with a value update; every result is checked
// against a host computation, and the exit status counts the failures.
#include <math.h>
#include <stdio.h>

#include "fastainv/droptol-tuning.h"
#include "fastainv/fastainv.h"
#include "formats/conversion.h"
#include "formats/formats.h"
#ifdef DRIVER_DEVICE
#include "cuda/spmv/kernel-iface.h"
#include "plan/plan.h"
#include "util/cuda/initialize.h"
#include "util/cuda/sblas.h"
#endif

template <class T> static csr_matrix<T> stencil(int L)
{
  // 7-point operator on an L^3 grid with position-dependent couplings
  csr_matrix<T> A;
  const int n = L * L * L;
  A.n_rows = A.n_cols = n;
  A.row_ptr.push_back(0);
  for (int z = 0; z < L; z++)
    for (int y = 0; y < L; y++)
      for (int x = 0; x < L; x++) {
        const int i = (z * L + y) * L + x;
        double diag = 1e-3;
        const int off[6][3] = {{0, 0, -1}, {0, -1, 0}, {-1, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        int cols[7];
        double vals[7];
        int k = 0;
        for (int d = 0; d < 6; d++) {
          const int zz = z + off[d][0], yy = y + off[d][1], xx = x + off[d][2];
          if (zz < 0 || yy < 0 || xx < 0 || zz >= L || yy >= L || xx >= L)
            continue;
          const int j = (zz * L + yy) * L + xx;
          const double w = 1.0 + 0.5 * sin(0.37 * (i + j));
          cols[k] = j;
          vals[k] = -w;
          diag += w;
          k++;
        }
        cols[k] = i;
        vals[k] = diag;
        k++;
        // insertion sort by column
        for (int a = 1; a < k; a++)
          for (int b = a; b > 0 && cols[b - 1] > cols[b]; b--) {
            int tc = cols[b];
            cols[b] = cols[b - 1];
            cols[b - 1] = tc;
            double tv = vals[b];
            vals[b] = vals[b - 1];
            vals[b - 1] = tv;
          }
        for (int a = 0; a < k; a++) {
          A.cols.push_back(cols[a]);
          A.elms.push_back((T)vals[a]);
        }
        A.row_ptr.push_back((int)A.cols.size());
      }
  A.n_nz = (int)A.cols.size();
  return A;
}

static unsigned long long fnv(const void *p, size_t bytes)
{
  unsigned long long h = 1469598103934665603ull;
  const unsigned char *c = (const unsigned char *)p;
  for (size_t k = 0; k < bytes; k++) {
    h ^= c[k];
    h *= 1099511628211ull;
  }
  return h;
}

template <class V> static unsigned long long hash(const V &v)
{
  return fnv(v.data(), v.size() * sizeof(v[0]));
}

template <class E> static void print_slell(const char *name, const slell_matrix<E, host_memory_space_tag> &B)
{
  printf("%s rows=%d cols=%d nz=%d S=%u slices=%u hblock=%u var=%d diags=%d sp=%zu:%016llx "
         "ci=%zu:%016llx el=%zu:%016llx\n",
         name, B.n_rows, B.n_cols, B.n_nz, B.slice_height, B.n_slices, B.hblock,
         (int)B.var_height, (int)B.diags, B.slice_ptr.size(), hash(B.slice_ptr), B.cols.size(),
         hash(B.cols), B.elms.size(), hash(B.elms));
}

template <class T> static void print_csr(const char *name, const csr_matrix<T> &G)
{
  printf("%s rows=%d nz=%d rp=%016llx ci=%016llx el=%016llx\n", name, G.n_rows, G.n_nz,
         hash(G.row_ptr), hash(G.cols), hash(G.elms));
}

static void count_rows(void *v) { ++*static_cast<long *>(v); }

static int failures = 0;
static void expect(bool ok, const char *what)
{
  printf("%s %s\n", what, ok ? "ok" : "FAILED");
  if (!ok)
    failures++;
}

int main()
{
  csr_matrix<double> A = stencil<double>(12);
  csr_matrix<float> A32 = stencil<float>(12);

  // the approximate inverse of the square system (before the conversions
  // below pad A's rows in place)
  long rows_done = 0;
  csr_matrix<double> G1, G2;
  const bool ok = fastainv_sym(G1, G2, A, count_rows, &rows_done, 1 << 22, 0.01);
  printf("fastainv double ok=%d progress=%ld\n", (int)ok, rows_done);
  print_csr("G1", G1);
  print_csr("G2", G2);
  csr_matrix<float> F1, F2;
  fastainv_sym(F1, F2, A, count_rows, &rows_done, 1 << 22, 0.05);
  print_csr("F1", F1);
  print_csr("F2", F2);

  slell_matrix<double, host_memory_space_tag> B = csr_to_slell(A, 32, 1, false, true);
  print_slell("diag32", B);
  slell_matrix<float, host_memory_space_tag> B2 = csr_to_slell(A32, 64, 2, false, false);
  print_slell("hblock64", B2);
  slell_matrix<float, host_memory_space_tag> B3 = csr_to_slell(A32, 64, 1, true, false);
  print_slell("var64", B3);
  csr_matrix<double> Ag = stencil<double>(10);
  slell_matrix<double, host_memory_space_tag> B4 = csr_to_slell_guess_format(Ag);
  print_slell("guess", B4);
  printf("padded rows=%d %d\n", A.n_rows, Ag.n_rows);

  DroptolTuner t;
  for (int k = 0; k < 14; k++) {
    if (k == 9)
      t.restart();
    const double d = t.getDroptol();
    const double l = log2(d) + 6.3;
    t.noteTime(1.0 + l * l);
    printf("tuner %d %.17g best %.17g it %d\n", k, d, t.getBestDroptol(), t.iterations());
  }

#ifdef DRIVER_DEVICE
  ispm_initialize();
  fprintf(stderr, "device %s\n", get_device_string().str);
  const int n = B.n_rows;  // padded
  vector<double, host_memory_space_tag> xh(n, 0.0);
  for (int i = 0; i < A.n_cols; i++)
    xh[i] = 0.25 * ((i * 7919) % 13 - 6);
  // host product of the padded CSR
  vector<double, host_memory_space_tag> yref(n, 0.0);
  for (int i = 0; i < A.n_rows; i++)
    for (int e = A.row_ptr[i]; e < A.row_ptr[i + 1]; e++)
      yref[i] += A.elms[e] * xh[A.cols[e]];
  double ynorm = 0;
  for (int i = 0; i < n; i++)
    ynorm = fmax(ynorm, fabs(yref[i]));
  auto close = [&](const vector<double, host_memory_space_tag> &y, double tol) {
    double e = 0;
    for (int i = 0; i < n; i++)
      e = fmax(e, fabs(y[i] - yref[i]));
    return e <= tol * ynorm;
  };

  slell_matrix<double, device_memory_space_tag> dB(B);
  vector<double, device_memory_space_tag> x(xh), y(n);
  spmv_launch_params p = {32, 32, 1, true, true};
  launch_spmv_kernel<double, double>(p, dB, x, y);
  vector<double, host_memory_space_tag> yh(y);
  expect(close(yh, 1e-14), "spmv<double,double> vector overload");
  spmv_launch_params p4 = {8, 32, 4, true, true};
  vector<double, device_memory_space_tag> y2(n);
  launch_spmv_kernel<double, double>(p4, dB, x.udata(), y2.udata());
  yh = y2;
  expect(close(yh, 1e-14), "spmv<double,double> pointer overload");
  {
    // the drop-in headers' stream overloads (no counterpart in the reference)
    cudaStream_t st;
    cudaStreamCreate(&st);
    vector<double, device_memory_space_tag> y5(n);
    launch_spmv_kernel<double, double>(p4, dB, x, y5, st);
    vector<double, device_memory_space_tag> s5(1);
    sblas::dot<double>(x.data(), y5.data(), s5.data(), n, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    vector<double, host_memory_space_tag> y5h(y5);
    expect(close(y5h, 1e-14), "spmv<double,double> on a stream");
  }
  // unsupported parameters launch nothing (y2 keeps its values)
  spmv_launch_params bad = {4, 32, 1, true, true};
  vector<double, device_memory_space_tag> y3(yh);
  launch_spmv_kernel<double, double>(bad, dB, x, y3);
  vector<double, host_memory_space_tag> y3h(y3);
  expect(close(y3h, 1e-14), "unsupported launch leaves y alone");

  slell_matrix<float, host_memory_space_tag> Bf = csr_to_slell(A32, 32, 1, false, true);
  slell_matrix<float, device_memory_space_tag> dBf(Bf);
  launch_spmv_kernel<double, float>(p, dBf, x, y);
  yh = y;
  expect(close(yh, 1e-6), "spmv<double,float>");

  vector<double, host_memory_space_tag> sh(1, 0.0);
  vector<double, device_memory_space_tag> s(1);
  sblas::dot<double>(x.data(), y.data(), s.data(), n);
  sh = s;
  double dref = 0, dabs = 0;
  for (int i = 0; i < n; i++) {
    dref += xh[i] * yh[i];
    dabs += fabs(xh[i] * yh[i]);
  }
  expect(fabs(sh[0] - dref) <= 1e-13 * dabs, "sblas::dot");

  vector<double, host_memory_space_tag> sc(5, 0.0);
  sc[2] = 3.0;  // gamma
  sc[3] = 2.0;  // gammaold
  sc[4] = 5.0;  // delta
  sc[0] = 0.5;  // alpha (previous)
  vector<double, device_memory_space_tag> dsc(sc);
  sblas::ppcg_update_scalars<double>(dsc.data(), dsc.data() + 1, dsc.data() + 2, dsc.data() + 3,
                                     dsc.data() + 4);
  sc = dsc;
  const double beta = 3.0 / 2.0, alpha = 3.0 / (5.0 - beta * 3.0 / 0.5);
  expect(sc[1] == beta && fabs(sc[0] - alpha) <= 1e-15 * fabs(alpha), "sblas::ppcg_update_scalars");

  vector<int, host_memory_space_tag> idx(4);
  idx[0] = 5;
  idx[1] = 1;
  idx[2] = 5;
  idx[3] = 0;
  vector<int, device_memory_space_tag> didx(idx);
  vector<double, device_memory_space_tag> g(4);
  sblas::copy_indexed<double>(g.data(), x.data(), didx.data(), 4);
  vector<double, host_memory_space_tag> gh(g);
  expect(gh[0] == xh[5] && gh[1] == xh[1] && gh[2] == xh[5] && gh[3] == xh[0],
         "sblas::copy_indexed");
  vector<double, host_memory_space_tag> acc(8, 0.0), src(4, 1.0);
  vector<double, device_memory_space_tag> dacc(acc), dsrc(src);
  sblas::add_indexed<double>(dacc.data(), dsrc.data(), didx.data(), 4);
  acc = dacc;
  expect(acc[5] == 2.0 && acc[1] == 1.0 && acc[0] == 1.0, "sblas::add_indexed");

  spmv_plan<double, double> plan(A, PLAN_DEFAULT);
  vector<double, device_memory_space_tag> y4(n);
  plan.execute_spmv(x, y4);
  yh = y4;
  expect(close(yh, 1e-14), "spmv_plan<double> DEFAULT");
  for (size_t k = 0; k < plan.host_matrix->elms.size(); k++)
    plan.host_matrix->elms[k] *= 2.0;
  plan.update_device_matrix_coefs();
  plan.execute_spmv(x.udata(), y4.udata());
  yh = y4;
  for (int i = 0; i < n; i++)
    yh[i] *= 0.5;
  expect(close(yh, 1e-14), "spmv_plan update_device_matrix_coefs");

  spmv_plan<float, float> planx(A32, PLAN_EXHAUSTIVE);
  vector<float, host_memory_space_tag> xf(n), yf(n);
  for (int i = 0; i < n; i++)
    xf[i] = (float)xh[i];
  vector<float, device_memory_space_tag> dxf(xf), dyf(n);
  planx.execute_spmv(dxf, dyf);
  yf = dyf;
  double ef = 0;
  for (int i = 0; i < n; i++)
    ef = fmax(ef, fabs((double)yf[i] - yref[i]));
  expect(ef <= 1e-5 * ynorm && planx.params.valid(), "spmv_plan<float> EXHAUSTIVE");
#endif
  printf("failures %d\n", failures);
  return failures ? 1 : 0;
}
