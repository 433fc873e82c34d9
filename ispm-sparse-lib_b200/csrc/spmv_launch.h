// Internal SpMV launch interface (used by the C ABI, the plan and the solver).
#ifndef ISPM_SPMV_LAUNCH_H
#define ISPM_SPMV_LAUNCH_H

#include <cuda_runtime.h>

#include "ispm_internal.h"

namespace ispm {

// Validate launch parameters against a matrix (no CUDA calls).
int check_launch(int x_dtype, const ispm_launch_params &p, const ispm_slell_view &m);
// Optional fused epilogue of an SpMV: *out = sum_i y_i v_i in FP64 over the
// rows the launch writes (v has the vector type T).  part holds one partial
// per CTA (part_capacity slots), ticket is a zero-initialised arrival counter
// the launch leaves at zero.
struct SpmvDot {
  const void *v = nullptr;
  double *out = nullptr;
  double *part = nullptr;
  unsigned *ticket = nullptr;
  unsigned part_capacity = 0;
  // optional second sum, *out2 = sum_i v_i^2 over the same rows (read in the
  // same pass); its partials go to part[part_capacity + CTA]
  double *out2 = nullptr;
};

// Batched solves (batch.cu).  The matrix is a block-diagonal stack of
// systems, each padded to whole 1024-row tiles; the vectors are a stack of
// lanes (a system's right-hand sides), also tile-padded.  The launch walks
// virtual tiles vt[0 .. n_vt): vt[k] = (matrix tile, lane tile), the matrix
// tile relative to this matrix, the lane tile a global vector tile; every CTA
// lies in one tile and reads x / writes y at its lane's rows, so all lanes
// of a system share one copy of its matrix (consecutive virtual tiles of a
// system's lanes reuse it from L2).  CTAs of lanes with done[lane] != 0
// return at once; with `out` set, out[lane] = sum of y_i v_i over the lane's
// rows (FP64), finished by the lane's last CTA to arrive: lane L's partials
// sit at part[cta_beg[L] .. cta_beg[L] + cta_cnt[L]) in tile order
// (lane_tile0[L]: the lane's first tile) and ticket[L] is a zero-initialised
// counter the launch leaves at zero.
struct SpmvLanes {
  const int *tile_lane = nullptr;  // lane of each tile (global tile index)
  unsigned tile_base = 0;          // global tile of the lanes' vector row 0
  const int2 *vt = nullptr;        // virtual tiles of the launch
  unsigned n_vt = 0;
  const int *lane_tile0 = nullptr;
  const int *done = nullptr;
  const void *v = nullptr;
  double *out = nullptr;
  double *part = nullptr;
  unsigned *ticket = nullptr;
  const int *cta_beg = nullptr;
  const int *cta_cnt = nullptr;
};

// FP16 elements (elm_dtype ISPM_F16) stored times a power of two: the launch
// computes y_i = inv_scale * (sum of the stored entries of row i times x),
// plus diag[i] * x[i] for a split operator (FP16 off-diagonal elements and
// an FP32 diagonal, one value per padded row, 0 past n_cols); diag NULL: no
// diagonal term (an FP16-stored factor).
struct SpmvSplit {
  const float *diag = nullptr;
  float inv_scale = 1.f;
};

// Tile records of the device matrix whose slice_ptr array is `slice_ptr`
// (registered by DeviceSlell uploads, dropped on release), the largest x
// area (words) and element count over its staged tiles.
struct StageInfo {
  const int *rec = nullptr;
  int max_x_words = 0;
  int max_elms = 0;
};
bool find_stage_records(const unsigned *slice_ptr, unsigned n_slices, StageInfo &out);

// Validate and launch y = A x on `s`.  `skip` (device int, may be NULL): the
// kernel returns at once when it holds a nonzero value.
// pdl: launch as a programmatic dependent of the stream's previous kernel
// (that kernel's results are read only after it completed; the matrix must
// be final before that kernel started, since the staged walk fetches its
// elements before the wait).
int launch_spmv(int x_dtype, const ispm_launch_params &p, const ispm_slell_view &m,
                const void *x, void *y, cudaStream_t s, const int *skip = nullptr,
                const SpmvDot *ep = nullptr, bool pdl = false,
                const SpmvSplit *split = nullptr);
// Lane-segmented launch (fixed slice height, T == E only; grid: n_vt tiles).
int launch_spmv_lanes(int x_dtype, const ispm_launch_params &p, const ispm_slell_view &m,
                      const void *x, void *y, cudaStream_t s, const SpmvLanes &lanes);
// CTAs a launch of matrix m with params p uses (partials a fused dot needs).
unsigned spmv_grid(const ispm_launch_params &p, const ispm_slell_view &m);
// Rows one CTA of such a launch covers (fixed slice height).
unsigned spmv_cta_rows(const ispm_launch_params &p, const ispm_slell_view &m);

// Device-resident sliced-ELL matrix.
// Staged diagonal walk (FP32 vectors, launch shape N = S, H = 1): the matrix
// is cut into tiles of kStageTileRows rows; every tile has a record of
// kStageRecInts ints, computed on the host from the slice records when a
// diagonal-block matrix of fixed slice height is uploaded.  A diagonal of
// slice s at diag_pos d serves tile row t = s S + r from x[w + t] with the
// window start w = d - S - s S; the tile's windows are the union of those
// starts over its slices (ascending, u = 0 .. nu - 1), merged into bands of
// x that a copy engine moves into shared memory beside the tile's elements
// (all of them: a tile's slices are consecutive in elms).  Ints [0, 152)
// travel to shared memory with the tile (the compute side), [152, 172) are
// the copy list the issuing warp reads:
//   [0] 0: not staged (the tile reads everything from global memory);
//       1: staged, every slice carries all nu windows in order (its k-th
//       diagonal is window k) and no explicit-column entries; 2: staged,
//       slices differ (masks below) or carry explicit-column entries.
//       Staged tiles have 1..64 window starts, every slice's diagonals in
//       ascending order and at most 8 bands;
//   [1] nu; [2] slices in the tile; [3..8) 0;
//   [8 + u] x-area word of x[w_u] (tile row t reads word [8 + u] + t);
//   [72 + 2s], [73 + 2s] slice s: bit u of this 64-bit mask is set when the
//       slice has a diagonal at window u (its k-th diagonal is its k-th set
//       bit);
//   [104 + s] slice s: offset of its first diagonal element from the tile's
//       first element;
//   [120 + s] slice s: explicit-column entries per row (its first element
//       sits that many times S before its first diagonal element);
//   [136 + s] slice s: its cols_end record (first column index, into cols);
//   [152] the tile's first element (index into elms), [153] its element
//       count; [154] nb, the number of bands; [155] x-area words;
//   [156 + 2q], [157 + 2q] band q: first x column (a multiple of 4, may be
//       negative), words (a multiple of 4); band q fills the x-area words
//       after bands 0 .. q-1; columns outside x read zero.
constexpr unsigned kStageTileRows = 256;
constexpr int kStageRecInts = 176;
constexpr int kStageRecComputeInts = 152;  // the part that travels with the tile
constexpr int kStageMaxBands = 8;
constexpr int kStageMaxDiag = 64;
constexpr int kStageMaxSlices = 16;        // slice height >= 16
constexpr int kStageMaxXWords = 8192;      // larger x areas are not staged
constexpr int kStageGap = 32;  // windows this close (in words) share a band

// Tile records of h (empty unless h is diagonal-block, fixed height, and its
// slice height divides kStageTileRows).
void stage_records(const HostSlell &h, std::vector<int> &rec);

struct DeviceSlell {
  ispm_slell_view meta{};  // host copy of the metadata; pointers are device pointers
  unsigned *slice_ptr = nullptr;
  unsigned *cols = nullptr;
  void *elms = nullptr;
  int *stage_rec = nullptr;  // tile records of the staged walk (device), or NULL
  // build, upload and register the tile records of h (no-op for other shapes)
  int attach_stage_records(const HostSlell &h);
  ispm_slell_view view() const
  {
    ispm_slell_view v = meta;
    v.slice_ptr = slice_ptr;
    v.cols = cols;
    v.elms = elms;
    return v;
  }
  // bf16_values: keep an FP32 element array as BF16 (elm_dtype ISPM_BF16)
  int upload(const HostSlell &h, bool bf16_values = false);
  // Keep an FP32 element array whose values are all exact binary16 values as
  // FP16 (elm_dtype ISPM_F16).
  int upload_f16(const HostSlell &h);
  int update_elms(const HostSlell &h);
  void release();
  ~DeviceSlell() { release(); }
};

// B200 launch heuristic for a matrix: threads per slice and rows per thread.
ispm_launch_params default_launch(int x_dtype, const ispm_slell_view &m);
// The same heuristic restricted to the register walk (several rows per
// thread, x gathered through the read-only path): the shapes the
// lane-segmented launches take.
ispm_launch_params register_walk_launch(int x_dtype, const ispm_slell_view &m);

// d.elms[map[k]] = vals[k] for k < n (device arrays; vals FP32 or FP64).
// Same from the slot side: d.elms[s] = vals[inv[s]] for every element slot
// s (0 where inv[s] < 0); writes are coalesced, reads stay within a slice's
// CSR range.
int refresh_values_gather(DeviceSlell &d, const int *inv, const void *vals, int val_dtype,
                          cudaStream_t s);
int refresh_values(DeviceSlell &d, const unsigned *map, const void *vals, int val_dtype,
                   long long n, cudaStream_t s);
// FP16 elements: d.elms[map[k]] = FP16(vals[k] * scale) (nearest).
int refresh_values_f16(DeviceSlell &d, const unsigned *map, const double *vals, long long n,
                       double scale, cudaStream_t s);
// out = max |vals[k]| over n device values (synchronous).
int device_absmax(const double *vals, long long n, double &out);

}  // namespace ispm

struct ispm_dslell {
  ispm::DeviceSlell d;
};

#endif
