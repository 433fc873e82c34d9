"""Python mirror of the ispm-sparse-lib hot-path API over the C ABI.

Names follow the reference's C++ API (formats/formats.h, formats/conversion.h,
plan/plan.h, fastainv/fastainv.h, cuda/spmv/kernel-iface.h, util/cuda/sblas.h,
fastainv/droptol-tuning.h, util/cuda/initialize.h) so that code written against
it reads like the reference's.  Everything computes in libispm_b200.so; this
module only marshals arguments.  Device vectors are passed as torch CUDA
tensors (device memory and streams only -- no torch kernels are used on the
path), or as raw device pointers (ints).

Error behaviour: every C-ABI status other than ISPM_OK raises IspmError; the
reference aborts on CUDA errors and silently ignores unsupported launch
parameters, both of which surface here as exceptions instead.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PKG = os.path.dirname(_HERE)
LIB_PATH = os.path.join(_PKG, "libispm_b200.so")

F32, F64 = 0, 1
BF16, F16 = 2, 3  # solver-internal element types
OK = 0
ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_ARCH = 1, 2, 3, 4
ERR_BREAKDOWN, ERR_NOT_CONVERGED, ERR_TIMEOUT, ERR_TOO_LARGE = 5, 6, 7, 8

PLAN_DEFAULT, PLAN_ESTIMATE, PLAN_EXHAUSTIVE = 0, 1, 2
SPMV_NO_TEXTURE_MEMORY, SPMV_PLAN_NO_DEVICE = 1, 2

_NP = {F32: np.float32, F64: np.float64}


class IspmError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class slell_view(C.Structure):
    _fields_ = [
        ("n_rows", C.c_int), ("n_cols", C.c_int), ("n_nz", C.c_int),
        ("slice_height", C.c_uint), ("n_slices", C.c_uint), ("hblock", C.c_uint),
        ("var_height", C.c_int), ("diags", C.c_int), ("elm_dtype", C.c_int),
        ("min_slice_height", C.c_uint), ("max_slice_height", C.c_uint),
        ("n_slice_ptr", C.c_longlong), ("n_cols_arr", C.c_longlong), ("n_elms", C.c_longlong),
        ("slice_ptr", C.c_void_p), ("cols", C.c_void_p), ("elms", C.c_void_p),
    ]


class slell_params(C.Structure):
    _fields_ = [("S", C.c_uint), ("H", C.c_uint), ("V", C.c_uint), ("D", C.c_uint)]


class spmv_launch_params(C.Structure):
    """cuda/spmv/kernel-iface.h:6-17"""
    _fields_ = [("N", C.c_uint), ("S", C.c_uint), ("H", C.c_uint),
                ("use_tex_sliceptr", C.c_int), ("use_tex_x", C.c_int)]

    def valid(self) -> bool:
        return bool(_lib().ispm_launch_params_valid(C.byref(self)))

    def __repr__(self):
        return f"spmv_launch_params(N={self.N}, S={self.S}, H={self.H})"


class fastainv_stats(C.Structure):
    _fields_ = [("storage_chunks", C.c_longlong), ("chunks_used", C.c_longlong),
                ("truncated_rows", C.c_longlong), ("breakdowns", C.c_longlong)]


_L = None


def _lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C {_PKG}` "
                "(there is no fallback implementation)")
        _L = C.CDLL(LIB_PATH)
        _declare(_L)
    return _L


def lib_handle():
    """The loaded libispm_b200.so (ctypes.CDLL)."""
    return _lib()


def _declare(L):
    vp, i, u, d, ll = C.c_void_p, C.c_int, C.c_uint, C.c_double, C.c_longlong
    ip = C.POINTER(C.c_int)
    sig = {
        "ispm_error_string": (C.c_char_p, [i]),
        "ispm_last_error": (C.c_char_p, []),
        "ispm_version": (C.c_char_p, []),
        "ispm_initialize": (i, []),
        "ispm_get_device_string": (i, [C.c_char_p, i]),
        "ispm_csr_to_slell": (i, [i, i, i, vp, vp, vp, i, i, i, i, i, C.POINTER(vp)]),
        "ispm_csr_to_slell_guess_format": (i, [i, i, i, vp, vp, vp, i, i, C.POINTER(vp)]),
        "ispm_slell_get_view": (i, [vp, C.POINTER(slell_view)]),
        "ispm_slell_elms": (vp, [vp]),
        "ispm_slell_spmv_bytes": (C.c_ulonglong, [vp, i, i]),
        "ispm_slell_free": (None, [vp]),
        "ispm_dslell_upload": (i, [vp, C.POINTER(vp)]),
        "ispm_dslell_upload_f16": (i, [vp, C.POINTER(vp)]),
        "ispm_slell_stage_records": (i, [vp, vp, C.c_longlong, C.POINTER(C.c_longlong)]),
        "ispm_spmv_stage_fault": (i, [C.POINTER(i)]),
        "ispm_dslell_update_elms": (i, [vp, vp]),
        "ispm_dslell_get_view": (i, [vp, C.POINTER(slell_view)]),
        "ispm_dslell_free": (None, [vp]),
        "ispm_launch_params_valid": (i, [C.POINTER(spmv_launch_params)]),
        "ispm_launch_spmv": (i, [i, C.POINTER(spmv_launch_params), C.POINTER(slell_view),
                                 vp, vp, vp]),
        "ispm_plan_create": (i, [i, i, i, i, vp, vp, vp, i, u, C.POINTER(vp)]),
        "ispm_plan_execute": (i, [vp, vp, vp, vp]),
        "ispm_plan_upload": (i, [vp]),
        "ispm_plan_update_device_matrix_coefs": (i, [vp]),
        "ispm_plan_change_host_matrix": (i, [vp, i, i, vp, vp, vp]),
        "ispm_plan_get_params": (i, [vp, C.POINTER(slell_params),
                                     C.POINTER(spmv_launch_params)]),
        "ispm_plan_host_matrix": (vp, [vp]),
        "ispm_plan_device_matrix": (vp, [vp]),
        "ispm_plan_tuned_seconds": (d, [vp]),
        "ispm_plan_free": (None, [vp]),
        "ispm_sblas_copy_indexed": (i, [i, vp, vp, vp, i, vp]),
        "ispm_sblas_add_indexed": (i, [i, vp, vp, vp, i, vp]),
        "ispm_sblas_dot": (i, [i, vp, vp, vp, i, vp]),
        "ispm_sblas_ppcg_update_scalars": (i, [i, vp, vp, vp, vp, vp, vp]),
        "ispm_sblas_ppcg_update_vectors": (i, [i] + [vp] * 15 + [i, vp]),
        "ispm_fastainv_sym": (i, [i, i, vp, vp, vp, vp, vp, ll, d, C.POINTER(vp),
                                  C.POINTER(vp), C.POINTER(fastainv_stats)]),
        "ispm_csr_get_info": (i, [vp, ip, ip, ip, ip]),
        "ispm_csr_get_arrays": (i, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
        "ispm_csr_free": (None, [vp]),
        "ispm_droptol_tuner_create": (vp, [d, d]),
        "ispm_droptol_tuner_get_droptol": (d, [vp]),
        "ispm_droptol_tuner_get_best_droptol": (d, [vp]),
        "ispm_droptol_tuner_note_time": (None, [vp, d]),
        "ispm_droptol_tuner_restart": (None, [vp]),
        "ispm_droptol_tuner_reset_phase": (None, [vp]),
        "ispm_droptol_tuner_iterations": (i, [vp]),
        "ispm_droptol_tuner_free": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _check(status: int):
    if status != OK:
        msg = _lib().ispm_last_error().decode() or _lib().ispm_error_string(status).decode()
        raise IspmError(status, msg)


def _ptr(a):
    """Address of a numpy array, torch tensor or raw int pointer."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(f"cannot take the address of {type(a)}")


def _dtype_code(a) -> int:
    if isinstance(a, np.ndarray):
        dt = a.dtype
    else:
        dt = getattr(a, "dtype", None)
    s = str(dt)
    if s.endswith("float32"):
        return F32
    if s.endswith("float64"):
        return F64
    raise TypeError(f"unsupported element type {dt}")


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


# ---------------------------------------------------------------------------
# util/cuda/initialize.h
# ---------------------------------------------------------------------------

def ispm_initialize():
    _check(_lib().ispm_initialize())


def get_device_string() -> str:
    buf = C.create_string_buffer(64)
    _check(_lib().ispm_get_device_string(buf, 64))
    return buf.value.decode()


def version() -> str:
    return _lib().ispm_version().decode()


# ---------------------------------------------------------------------------
# formats/formats.h
# ---------------------------------------------------------------------------

class csr_matrix:
    """formats/formats.h:18-37 (host CSR): row_ptr int32[n+1], cols int32[nnz],
    elms float32/float64[nnz]."""

    def __init__(self, n_rows, n_cols, row_ptr, cols, elms):
        self.n_rows = int(n_rows)
        self.n_cols = int(n_cols)
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)
        self.elms = np.ascontiguousarray(elms)
        if self.elms.dtype not in (np.float32, np.float64):
            self.elms = self.elms.astype(np.float64)
        self.n_nz = int(self.row_ptr[-1])

    def pad(self, k: int):
        """formats.h:23-30: append empty rows up to a multiple of k (in place)."""
        n_pad = (self.n_rows + k - 1) // k * k
        if n_pad > self.n_rows:
            self.row_ptr = np.concatenate(
                [self.row_ptr, np.full(n_pad - self.n_rows, self.row_ptr[-1], np.int32)])
            self.n_rows = n_pad

    def spmv_bytes(self) -> int:
        """formats.h:32-36"""
        return 4 * (self.row_ptr.size + self.cols.size) + self.elms.itemsize * (
            self.elms.size + 2 * self.n_rows)

    def astype(self, dtype):
        return csr_matrix(self.n_rows, self.n_cols, self.row_ptr, self.cols,
                          self.elms.astype(dtype))

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.elms, self.cols, self.row_ptr),
                             shape=(self.n_rows, self.n_cols))


class slell_matrix:
    """Host sliced-ELL matrix (formats/formats.h:44-102), owned by the library."""

    def __init__(self, handle, owner=True, keepalive=None):
        self._h = C.c_void_p(handle)
        self._owner = owner
        self._keep = keepalive

    def __del__(self):
        if getattr(self, "_owner", False) and self._h and _L is not None:
            _L.ispm_slell_free(self._h)
            self._h = None

    def view(self) -> slell_view:
        v = slell_view()
        _check(_lib().ispm_slell_get_view(self._h, C.byref(v)))
        return v

    def __getattr__(self, name):
        if name in ("n_rows", "n_cols", "n_nz", "slice_height", "n_slices", "hblock",
                    "var_height", "diags", "elm_dtype", "min_slice_height",
                    "max_slice_height"):
            return getattr(self.view(), name)
        raise AttributeError(name)

    def _arr(self, ptr, n, dtype):
        if n == 0:
            return np.zeros(0, dtype)
        buf = (C.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr)
        return np.frombuffer(buf, dtype=dtype, count=n)

    @property
    def slice_ptr(self):
        v = self.view()
        return self._arr(v.slice_ptr, v.n_slice_ptr, np.uint32).copy()

    @property
    def cols(self):
        v = self.view()
        return self._arr(v.cols, v.n_cols_arr, np.uint32).copy()

    @property
    def elms(self):
        """Live (writable) view of the host element array."""
        v = self.view()
        return self._arr(_lib().ispm_slell_elms(self._h), v.n_elms, _NP[v.elm_dtype])

    def spmv_bytes(self, effective=False, vec_elt_size=None):
        v = self.view()
        if vec_elt_size is None:
            vec_elt_size = 4 if v.elm_dtype == F32 else 8
        return int(_lib().ispm_slell_spmv_bytes(self._h, int(effective), int(vec_elt_size)))

    def upload(self) -> "device_slell_matrix":
        """slell_matrix<E, device>(host) (formats.h:56-66)."""
        out = C.c_void_p()
        _check(_lib().ispm_dslell_upload(self._h, C.byref(out)))
        return device_slell_matrix(out.value, owner=True)

    def upload_f16(self) -> "device_slell_matrix":
        """Device copy with FP16 elements (every FP32 element must be an exact
        binary16 value, as in an FP16 split)."""
        out = C.c_void_p()
        _check(_lib().ispm_dslell_upload_f16(self._h, C.byref(out)))
        return device_slell_matrix(out.value, owner=True)

    def stage_records(self) -> np.ndarray:
        """Tile records of the staged SpMV walk (176 ints per 256-row tile)."""
        L = _lib()
        n = C.c_longlong()
        _check(L.ispm_slell_stage_records(self._h, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), np.int32)
        _check(L.ispm_slell_stage_records(self._h, _ptr(out), n.value, C.byref(n)))
        return out[: n.value].reshape(-1, 176) if n.value else out[:0].reshape(0, 176)


class device_slell_matrix:
    """Device sliced-ELL matrix (slell_matrix<E, device_memory_space_tag>)."""

    def __init__(self, handle, owner=True, keepalive=None):
        self._h = C.c_void_p(handle)
        self._owner = owner
        self._keep = keepalive

    def __del__(self):
        if getattr(self, "_owner", False) and self._h and _L is not None:
            _L.ispm_dslell_free(self._h)
            self._h = None

    def view(self) -> slell_view:
        v = slell_view()
        _check(_lib().ispm_dslell_get_view(self._h, C.byref(v)))
        return v

    def update_elms(self, host: slell_matrix):
        _check(_lib().ispm_dslell_update_elms(self._h, host._h))

    def __getattr__(self, name):
        if name in ("n_rows", "n_cols", "n_nz", "slice_height", "n_slices", "hblock",
                    "var_height", "diags", "elm_dtype", "min_slice_height",
                    "max_slice_height"):
            return getattr(self.view(), name)
        raise AttributeError(name)


# ---------------------------------------------------------------------------
# formats/conversion.h
# ---------------------------------------------------------------------------

def csr_to_slell(A: csr_matrix, req_slice_height: int, hblock: int, var_height: bool,
                 use_diags: bool, min_height: int = 4) -> slell_matrix:
    """conversion.h:338-414.  Like the reference, pads A to a multiple of 512
    rows in place (conversion.h:343)."""
    code = _dtype_code(A.elms)
    out = C.c_void_p()
    _check(_lib().ispm_csr_to_slell(code, A.n_rows, A.n_cols, _ptr(A.row_ptr), _ptr(A.cols),
                                    _ptr(A.elms), int(req_slice_height), int(hblock),
                                    int(bool(var_height)), int(bool(use_diags)),
                                    int(min_height), C.byref(out)))
    A.pad(512)
    return slell_matrix(out.value)


def csr_to_slell_guess_format(A: csr_matrix, examine_ratio: int = 1,
                              min_height: int = 4) -> slell_matrix:
    """conversion.h:416-492"""
    code = _dtype_code(A.elms)
    out = C.c_void_p()
    _check(_lib().ispm_csr_to_slell_guess_format(code, A.n_rows, A.n_cols, _ptr(A.row_ptr),
                                                 _ptr(A.cols), _ptr(A.elms),
                                                 int(examine_ratio), int(min_height),
                                                 C.byref(out)))
    A.pad(512)
    return slell_matrix(out.value)


# ---------------------------------------------------------------------------
# cuda/spmv/kernel-iface.h
# ---------------------------------------------------------------------------

def launch_spmv_kernel(params: spmv_launch_params, m, x, y, stream=None):
    """launch_spmv_kernel<T, E>(params, m, x, y): T from x's dtype, E from m."""
    v = m.view() if hasattr(m, "view") else m
    _check(_lib().ispm_launch_spmv(_dtype_code(x), C.byref(params), C.byref(v), _ptr(x),
                                   _ptr(y), _stream(stream)))


def solver_shape(A: csr_matrix, elm_dtype=np.float32) -> tuple:
    """(S, hblock, var_height, diags): the shape the solver stores the n x n
    operator A in with elm_dtype elements (ispm_solver_choose_shape)."""
    L = _lib()
    L.ispm_solver_choose_shape.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.POINTER(slell_params)]
    L.ispm_solver_choose_shape.restype = C.c_int
    v = np.ascontiguousarray(A.elms, np.float64)
    p = slell_params()
    _check(L.ispm_solver_choose_shape(F32 if np.dtype(elm_dtype) == np.float32 else F64,
                                      A.n_rows, _ptr(A.row_ptr), _ptr(A.cols), _ptr(v),
                                      C.byref(p)))
    return (p.S, p.H, p.V, p.D)


def rcm_order(A: csr_matrix) -> np.ndarray:
    """Reverse Cuthill-McKee ordering of A's (symmetric) pattern: perm[new] = old."""
    L = _lib()
    L.ispm_rcm_order.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.ispm_rcm_order.restype = C.c_int
    perm = np.zeros(max(A.n_rows, 1), np.int32)
    _check(L.ispm_rcm_order(A.n_rows, _ptr(A.row_ptr), _ptr(A.cols), _ptr(perm)))
    return perm[: A.n_rows]


def csr_bandwidth(A: csr_matrix) -> int:
    """max |col - row| over A's pattern."""
    L = _lib()
    L.ispm_csr_bandwidth.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
    L.ispm_csr_bandwidth.restype = C.c_longlong
    bw = L.ispm_csr_bandwidth(A.n_rows, _ptr(A.row_ptr), _ptr(A.cols))
    if bw < 0:
        _check(ERR_INVALID)
    return int(bw)


def permute_symmetric(A: csr_matrix, perm: np.ndarray) -> csr_matrix:
    """P A P^T with perm[new] = old (rows and columns renumbered, columns
    sorted within each row)."""
    import scipy.sparse as sp
    M = sp.csr_matrix((A.elms, A.cols, A.row_ptr), shape=(A.n_rows, A.n_cols))
    M = M[perm][:, perm].tocsr()
    M.sort_indices()
    return csr_matrix(A.n_rows, A.n_cols, M.indptr.astype(np.int32),
                      M.indices.astype(np.int32), M.data.astype(A.elms.dtype))


def csr_split_f16(A: csr_matrix):
    """The FP16 split the solver's matrix_f16 option stores: (off, diag,
    scale) with off[k] the binary16 bit pattern (uint16) of A's CSR entry k
    times scale (0 on diagonal entries) and diag the FP32 diagonal corrected
    by the rounding of the row's off-diagonal magnitudes."""
    L = _lib()
    vp = C.c_void_p
    L.ispm_csr_split_f16.argtypes = [C.c_int, vp, vp, vp, vp, vp, C.POINTER(C.c_float)]
    L.ispm_csr_split_f16.restype = C.c_int
    n = A.row_ptr.size - 1
    vals = np.ascontiguousarray(A.elms, np.float64)
    off = np.zeros(max(int(A.row_ptr[n]), 1), np.uint16)
    diag = np.zeros(max(n, 1), np.float32)
    sc = C.c_float()
    _check(L.ispm_csr_split_f16(n, _ptr(A.row_ptr), _ptr(A.cols), _ptr(vals), _ptr(off),
                                _ptr(diag), C.byref(sc)))
    return off[: int(A.row_ptr[n])], diag[:n], float(sc.value)


class device_split_f16:
    """Device copy of the FP16 split of an FP64 CSR A (csr_split_f16): the
    off-diagonal part as sliced-ELL with binary16 elements (shape `fmt` =
    (S, hblock, var_height, diags), or the reference's guess), the FP32
    diagonal (n_rows padded entries) and 1 / scale.  Device arrays are torch
    tensors; `view` describes them for launch_spmv_split."""

    def __init__(self, A: csr_matrix, fmt=None):
        import torch
        off, diag, sc = csr_split_f16(A)
        n = A.row_ptr.size - 1
        rows = np.repeat(np.arange(n), np.diff(A.row_ptr))
        keep = A.cols != rows
        orp = np.zeros(n + 1, np.int32)
        orp[1:] = np.cumsum(np.bincount(rows[keep], minlength=n))
        vals = off.view(np.float16)[keep].astype(np.float32)
        Ao = csr_matrix(n, n, orp, np.ascontiguousarray(A.cols[keep], np.int32), vals)
        self.host = csr_to_slell_guess_format(Ao) if fmt is None else csr_to_slell(Ao, *fmt)
        v = self.host.view()
        # the library's FP16 upload (it checks every value is a binary16 value)
        self.dev = self.host.upload_f16()
        dg = np.zeros(v.n_rows, np.float32)
        dg[:n] = diag
        self.diag = torch.from_numpy(dg).to(torch.device("cuda"))
        self.scale = sc
        self.inv_scale = 1.0 / sc
        self.view_ = self.dev.view()

    def view(self) -> slell_view:
        return self.view_

    def bytes(self) -> int:
        """Stored bytes: slice_ptr + cols + FP16 elements + FP32 diagonal."""
        v = self.view_
        return 4 * v.n_slice_ptr + 4 * v.n_cols_arr + 2 * v.n_elms + 4 * v.n_rows

    def apply(self, params: spmv_launch_params, x, y, stream=None):
        launch_spmv_split(params, self.view_, self.diag, self.inv_scale, x, y, stream)


def launch_spmv_split(params: spmv_launch_params, view: slell_view, diag, inv_scale: float,
                      x, y, stream=None):
    """y = inv_scale * (A_off x) + diag * x: `view` describes the off-diagonal
    part with FP16 elements (elm_dtype F16) in device memory; diag None:
    y = inv_scale * (A x) (an FP16-stored factor)."""
    L = _lib()
    vp = C.c_void_p
    L.ispm_launch_spmv_split.argtypes = [C.POINTER(spmv_launch_params), C.POINTER(slell_view),
                                         vp, C.c_float, vp, vp, vp]
    L.ispm_launch_spmv_split.restype = C.c_int
    _check(L.ispm_launch_spmv_split(C.byref(params), C.byref(view), _ptr(diag),
                                    float(inv_scale), _ptr(x), _ptr(y), _stream(stream)))


def spmv_stage_fault() -> int:
    """The staged SpMV walk's wait-timeout record since the last call (0:
    none; 1 a compute warp's wait, 2 the copy warp's wait), cleared by the
    call."""
    code = C.c_int()
    _check(_lib().ispm_spmv_stage_fault(C.byref(code)))
    return code.value


# ---------------------------------------------------------------------------
# plan/plan.h
# ---------------------------------------------------------------------------

class spmv_plan:
    """spmv_plan<T, E> (plan/plan.h:20-161).  T is the vector type, E the
    matrix element type (taken from the CSR)."""

    def __init__(self, m: csr_matrix, kind: int = PLAN_DEFAULT, flags: int = 0, T=None):
        edt = _dtype_code(m.elms)
        vdt = edt if T is None else (F64 if np.dtype(T) == np.float64 else F32)
        out = C.c_void_p()
        _check(_lib().ispm_plan_create(vdt, edt, m.n_rows, m.n_cols, _ptr(m.row_ptr),
                                       _ptr(m.cols), _ptr(m.elms), int(kind), int(flags),
                                       C.byref(out)))
        self._h = out
        self.vec_dtype = vdt
        self.elm_dtype = edt

    def __del__(self):
        if getattr(self, "_h", None) and _L is not None:
            _L.ispm_plan_free(self._h)
            self._h = None

    def execute_spmv(self, x, y, stream=None):
        _check(_lib().ispm_plan_execute(self._h, _ptr(x), _ptr(y), _stream(stream)))

    def upload(self):
        _check(_lib().ispm_plan_upload(self._h))

    def update_device_matrix_coefs(self):
        _check(_lib().ispm_plan_update_device_matrix_coefs(self._h))

    def change_host_matrix(self, m: csr_matrix):
        _check(_lib().ispm_plan_change_host_matrix(self._h, m.n_rows, m.n_cols,
                                                   _ptr(m.row_ptr), _ptr(m.cols),
                                                   _ptr(m.elms)))

    @property
    def mparams(self) -> slell_params:
        mp, p = slell_params(), spmv_launch_params()
        _check(_lib().ispm_plan_get_params(self._h, C.byref(mp), C.byref(p)))
        return mp

    @property
    def params(self) -> spmv_launch_params:
        mp, p = slell_params(), spmv_launch_params()
        _check(_lib().ispm_plan_get_params(self._h, C.byref(mp), C.byref(p)))
        return p

    @property
    def host_matrix(self):
        h = _lib().ispm_plan_host_matrix(self._h)
        return slell_matrix(h, owner=False, keepalive=self) if h else None

    @property
    def device_matrix(self):
        h = _lib().ispm_plan_device_matrix(self._h)
        return device_slell_matrix(h, owner=False, keepalive=self) if h else None

    @property
    def tuned_seconds(self) -> float:
        return float(_lib().ispm_plan_tuned_seconds(self._h))


# ---------------------------------------------------------------------------
# fastainv/fastainv.h
# ---------------------------------------------------------------------------

_PROGRESS = C.CFUNCTYPE(None, C.c_void_p)


def _csr_from_handle(h) -> csr_matrix:
    L = _lib()
    nr, nc, nz, dt = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    _check(L.ispm_csr_get_info(h, C.byref(nr), C.byref(nc), C.byref(nz), C.byref(dt)))
    rp, ci, el = C.c_void_p(), C.c_void_p(), C.c_void_p()
    _check(L.ispm_csr_get_arrays(h, C.byref(rp), C.byref(ci), C.byref(el)))
    n, nnz = nr.value, nz.value
    npdt = _NP[dt.value]

    def arr(p, count, t):
        if count == 0:
            return np.zeros(0, t)
        return np.frombuffer((C.c_char * (count * np.dtype(t).itemsize)).from_address(p),
                             dtype=t, count=count).copy()

    out = csr_matrix(n, nc.value, arr(rp.value, n + 1, np.int32), arr(ci.value, nnz, np.int32),
                     arr(el.value, nnz, npdt))
    L.ispm_csr_free(h)
    return out


def fastainv_sym(A: csr_matrix, out_dtype=np.float64, progress=None,
                 max_elts: int = 8192000, droptol: float = 0.125, stats=None):
    """fastainv_sym<double, out_real>(Ainv1, Ainv2, A, progress, v, max_elts,
    droptol) (fastainv/fastainv.h:8-30).  Returns (Ainv1, Ainv2)."""
    if A.elms.dtype != np.float64:
        raise TypeError("fastainv_sym takes an FP64 CSR (csr_matrix<double>)")
    odt = F64 if np.dtype(out_dtype) == np.float64 else F32
    cb = _PROGRESS(lambda _v: progress()) if progress else None
    g1, g2 = C.c_void_p(), C.c_void_p()
    st = fastainv_stats()
    _check(_lib().ispm_fastainv_sym(odt, A.n_rows, _ptr(A.row_ptr), _ptr(A.cols),
                                    _ptr(A.elms), C.cast(cb, C.c_void_p) if cb else None,
                                    None, int(max_elts), float(droptol), C.byref(g1),
                                    C.byref(g2), C.byref(st)))
    if stats is not None:
        stats.update({k: getattr(st, k) for k, _ in fastainv_stats._fields_})
    return _csr_from_handle(g1), _csr_from_handle(g2)


# ---------------------------------------------------------------------------
# fastainv/droptol-tuning.h
# ---------------------------------------------------------------------------

class DroptolTuner:
    def __init__(self, lo: float = -10, hi: float = -3):
        self._h = C.c_void_p(_lib().ispm_droptol_tuner_create(float(lo), float(hi)))

    def __del__(self):
        if getattr(self, "_h", None) and _L is not None:
            _L.ispm_droptol_tuner_free(self._h)
            self._h = None

    def getDroptol(self) -> float:
        return _lib().ispm_droptol_tuner_get_droptol(self._h)

    def getBestDroptol(self) -> float:
        return _lib().ispm_droptol_tuner_get_best_droptol(self._h)

    def noteTime(self, t: float):
        _lib().ispm_droptol_tuner_note_time(self._h, float(t))

    def restart(self):
        _lib().ispm_droptol_tuner_restart(self._h)

    def resetPhase(self):
        _lib().ispm_droptol_tuner_reset_phase(self._h)

    def iterations(self) -> int:
        return _lib().ispm_droptol_tuner_iterations(self._h)


# ---------------------------------------------------------------------------
# util/cuda/sblas.h (device pointers / CUDA tensors)
# ---------------------------------------------------------------------------

class sblas:
    @staticmethod
    def copy_indexed(dst, src, i, n_elts, stream=None):
        _check(_lib().ispm_sblas_copy_indexed(_dtype_code(dst), _ptr(dst), _ptr(src), _ptr(i),
                                              int(n_elts), _stream(stream)))

    @staticmethod
    def add_indexed(dst, src, i, n_elts, stream=None):
        _check(_lib().ispm_sblas_add_indexed(_dtype_code(dst), _ptr(dst), _ptr(src), _ptr(i),
                                             int(n_elts), _stream(stream)))

    @staticmethod
    def dot(x, y, s, n_elts, stream=None):
        _check(_lib().ispm_sblas_dot(_dtype_code(x), _ptr(x), _ptr(y), _ptr(s), int(n_elts),
                                     _stream(stream)))

    @staticmethod
    def ppcg_update_scalars(alpha, beta, gamma, gammaold, delta, stream=None):
        _check(_lib().ispm_sblas_ppcg_update_scalars(
            _dtype_code(alpha), _ptr(alpha), _ptr(beta), _ptr(gamma), _ptr(gammaold),
            _ptr(delta), _stream(stream)))

    @staticmethod
    def ppcg_update_vectors(resnorm, gamma, delta, alpha, beta, n, m, p, s, q, z, x, r, u, w,
                            n_elts, stream=None):
        _check(_lib().ispm_sblas_ppcg_update_vectors(
            _dtype_code(x), _ptr(resnorm), _ptr(gamma), _ptr(delta), _ptr(alpha), _ptr(beta),
            _ptr(n), _ptr(m), _ptr(p), _ptr(s), _ptr(q), _ptr(z), _ptr(x), _ptr(r), _ptr(u),
            _ptr(w), int(n_elts), _stream(stream)))


# ---------------------------------------------------------------------------
# Pipelined PCG with FP64 refinement (the loop of the reference's external
# solver driver, composed from the primitives above)
# ---------------------------------------------------------------------------

class solver_opts(C.Structure):
    _fields_ = [("inner_dtype", C.c_int), ("tol", C.c_double), ("max_iters", C.c_int),
                ("max_refinements", C.c_int), ("check_every", C.c_int),
                ("use_graph", C.c_int), ("replace_ratio_f32", C.c_double),
                ("replace_ratio_f64", C.c_double), ("variant", C.c_int), ("prec", C.c_int),
                ("factor_bf16", C.c_int), ("reorder", C.c_int), ("matrix_f16", C.c_int),
                ("factor_f16", C.c_int), ("refresh", C.c_int)]


class solve_stats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("refinements", C.c_int), ("converged", C.c_int),
                ("status", C.c_int), ("true_relres", C.c_double), ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_SOLVER_DECLARED = False


def _declare_solver():
    global _SOLVER_DECLARED
    if _SOLVER_DECLARED:
        return
    L = _lib()
    vp, i = C.c_void_p, C.c_int
    L.ispm_solver_default_opts.argtypes = [C.POINTER(solver_opts)]
    L.ispm_solver_default_opts.restype = None
    L.ispm_solver_create.argtypes = [i, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                     C.POINTER(solver_opts), C.POINTER(vp)]
    L.ispm_solver_create.restype = i
    L.ispm_solver_rows.argtypes = [vp]
    L.ispm_solver_rows.restype = i
    L.ispm_solver_solve.argtypes = [vp, vp, vp, C.POINTER(solve_stats), vp]
    L.ispm_solver_solve.restype = i
    L.ispm_solver_solve_host.argtypes = [vp, vp, vp, C.POINTER(solve_stats), vp]
    L.ispm_solver_solve_host.restype = i
    L.ispm_solver_history.argtypes = [vp, vp, i]
    L.ispm_solver_history.restype = i
    L.ispm_solver_free.argtypes = [vp]
    L.ispm_solver_free.restype = None
    L.ispm_solver_update_values.argtypes = [vp, vp, i]
    L.ispm_solver_update_values.restype = i
    _SOLVER_DECLARED = True


class PCGSolver:
    """Preconditioned pipelined CG with FP64 iterative refinement.

    A: FP64 csr_matrix (SPD).  G1, G2: the fastainv_sym pair (Ainv1, Ainv2) or
    None.  inner: np.float64 (plain FP64) or np.float32 (mixed precision: FP32
    matrices / vectors, FP64 reductions).  Reliable updates recompute the
    true residual with the FP64 matrix whenever the recursive residual has
    fallen by replace_ratio since the previous one.  matrix_f16 (FP32 inner
    only): the inner iterations use the FP16 split of A (csr_split_f16).
    refresh: keep the maps update_values needs (new values of A, same
    pattern, rewritten on the device).  use_graph: True (1) replays chunks of
    check_every iterations as a CUDA graph, 2 runs the chunk inside the
    graph's while node until the device flags end the phase (classic
    iteration), False launches eagerly."""

    def __init__(self, A: csr_matrix, G1: csr_matrix | None = None,
                 G2: csr_matrix | None = None, inner=np.float32, tol: float = 1e-10,
                 max_iters: int = 100000, max_refinements: int = 500,
                 check_every: int = 16, use_graph: bool | int = True,
                 replace_ratio: float | None = None, variant: str = "auto",
                 prec: str = "given", factor_bf16: bool = False, reorder: str = "auto",
                 matrix_f16: bool = False, factor_f16: bool | None = None,
                 refresh: bool = False):
        _declare_solver()
        L = _lib()
        o = solver_opts()
        L.ispm_solver_default_opts(C.byref(o))
        o.inner_dtype = F64 if np.dtype(inner) == np.float64 else F32
        o.tol, o.max_iters, o.max_refinements = tol, max_iters, max_refinements
        o.check_every, o.use_graph = check_every, int(use_graph)
        if replace_ratio is not None:
            o.replace_ratio_f32 = o.replace_ratio_f64 = replace_ratio
        o.variant = {"auto": 0, "pipelined": 1, "classic": 2}[variant]
        o.prec = {"given": 0, "fsai_gpu": 1}[prec]
        o.factor_bf16 = int(factor_bf16)
        o.reorder = {"none": 0, "rcm": 1, "auto": 2}[reorder]
        o.matrix_f16 = int(matrix_f16)
        if factor_f16 is not None:  # None: the library default (on)
            o.factor_f16 = int(factor_f16)
        o.refresh = int(refresh)
        if A.elms.dtype != np.float64:
            raise TypeError("the solver takes the FP64 matrix")
        self._keep = [A, G1, G2]
        out = C.c_void_p()
        G1e = None if G1 is None else np.ascontiguousarray(G1.elms, np.float64)
        G2e = None if G2 is None else np.ascontiguousarray(G2.elms, np.float64)
        self._keep += [G1e, G2e]
        args = [A.n_rows, _ptr(A.row_ptr), _ptr(A.cols), _ptr(A.elms),
                None if G1 is None else _ptr(G1.row_ptr), None if G1 is None else _ptr(G1.cols),
                None if G1 is None else _ptr(G1e),
                None if G2 is None else _ptr(G2.row_ptr), None if G2 is None else _ptr(G2.cols),
                None if G2 is None else _ptr(G2e)]
        _check(L.ispm_solver_create(*args, C.byref(o), C.byref(out)))
        self._h = out
        self.n = A.n_rows
        self.opts = o

    def __del__(self):
        if getattr(self, "_h", None) and _L is not None:
            _L.ispm_solver_free(self._h)
            self._h = None

    @property
    def rows(self) -> int:
        return int(_lib().ispm_solver_rows(self._h))

    def _finish(self, status, st):
        if status not in (OK, ERR_NOT_CONVERGED, ERR_BREAKDOWN):
            _check(status)
        return st.as_dict()

    def solve(self, b, x, stream=None) -> dict:
        """b, x: FP64 device vectors of `rows` entries (torch tensors or pointers)."""
        st = solve_stats()
        rc = _lib().ispm_solver_solve(self._h, _ptr(b), _ptr(x), C.byref(st), _stream(stream))
        return self._finish(rc, st)

    def solve_host(self, b: np.ndarray, stream=None, out: np.ndarray | None = None):
        """Host vectors: copies b in and x out inside the call (into `out` when
        given, e.g. a pinned buffer).  Returns (x, stats)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.n) if out is None else out
        assert x.dtype == np.float64 and x.flags.c_contiguous and x.size >= self.n
        st = solve_stats()
        rc = _lib().ispm_solver_solve_host(self._h, _ptr(b), _ptr(x), C.byref(st),
                                           _stream(stream))
        return x, self._finish(rc, st)

    def history(self):
        buf = np.zeros(256)
        k = _lib().ispm_solver_history(self._h, _ptr(buf), 256)
        return buf[: min(k, 256)].copy()

    def operator(self, which: int = 0):
        """(view, launch params) of the device matrix the solver iterates
        with: 0 inner A, 1 FP64 A, 2 G, 3 G^T."""
        L = _lib()
        L.ispm_solver_operator.argtypes = [C.c_void_p, C.c_int, C.POINTER(slell_view),
                                           C.POINTER(spmv_launch_params)]
        L.ispm_solver_operator.restype = C.c_int
        v, p = slell_view(), spmv_launch_params()
        _check(L.ispm_solver_operator(self._h, which, C.byref(v), C.byref(p)))
        return v, p

    def update_values(self, vals) -> None:
        """New FP64 values of A in the CSR order given at construction: a numpy
        array (host) or a CUDA tensor (device).  Needs refresh=True."""
        on_dev = not isinstance(vals, np.ndarray)
        if not on_dev:
            vals = np.ascontiguousarray(vals, np.float64)
        _check(_lib().ispm_solver_update_values(self._h, _ptr(vals), int(on_dev)))


def default_launch_params(m, x_dtype=None) -> spmv_launch_params:
    """The launch shape the DEFAULT plan uses for matrix m (host or device)."""
    L = _lib()
    L.ispm_default_launch.argtypes = [C.c_int, C.POINTER(slell_view),
                                      C.POINTER(spmv_launch_params)]
    L.ispm_default_launch.restype = C.c_int
    v = m.view() if hasattr(m, "view") else m
    if x_dtype is None:
        x_dtype = v.elm_dtype
    elif not isinstance(x_dtype, int):
        x_dtype = F64 if np.dtype(x_dtype) == np.float64 else F32
    p = spmv_launch_params()
    _check(L.ispm_default_launch(int(x_dtype), C.byref(v), C.byref(p)))
    return p


def slell_value_map(m: slell_matrix, A: csr_matrix) -> np.ndarray:
    """map[k] = element slot of CSR entry k of A in the sliced-ELL matrix m
    (converted from a CSR with A's pattern)."""
    L = _lib()
    vp = C.c_void_p
    L.ispm_slell_value_map.argtypes = [vp, C.c_int, vp, vp, vp]
    L.ispm_slell_value_map.restype = C.c_int
    out = np.zeros(max(A.n_nz, 1), np.uint32)
    n_src = A.row_ptr.size - 1
    _check(L.ispm_slell_value_map(m._h, n_src, _ptr(A.row_ptr), _ptr(A.cols), _ptr(out)))
    return out[: A.n_nz]


def plan_refresh_values(plan: "spmv_plan", A: csr_matrix, vals_dev, stream=None):
    """Scatter new CSR values (device array, A's pattern) into the plan's device
    matrix (ispm_plan_refresh_values)."""
    L = _lib()
    vp = C.c_void_p
    L.ispm_plan_refresh_values.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int, vp]
    L.ispm_plan_refresh_values.restype = C.c_int
    n_src = A.row_ptr.size - 1
    _check(L.ispm_plan_refresh_values(plan._h, n_src, _ptr(A.row_ptr), _ptr(A.cols),
                                      _ptr(vals_dev), _dtype_code(vals_dev), _stream(stream)))


def fsai_sym_gpu(A: csr_matrix, out_dtype=np.float64, stats=None):
    """FSAI pair built on the GPU (ispm_fsai_sym_gpu): (Ainv1, Ainv2) = (G, G^T)
    with G lower triangular on A's lower pattern; Ainv2 Ainv1 ~ A^-1."""
    L = _lib()
    vp = C.c_void_p
    L.ispm_fsai_sym_gpu.argtypes = [C.c_int, C.c_int, vp, vp, vp, C.POINTER(vp),
                                    C.POINTER(vp), C.POINTER(C.c_uint)]
    L.ispm_fsai_sym_gpu.restype = C.c_int
    odt = F64 if np.dtype(out_dtype) == np.float64 else F32
    g1, g2, fb = C.c_void_p(), C.c_void_p(), C.c_uint()
    _check(L.ispm_fsai_sym_gpu(odt, A.n_rows, _ptr(A.row_ptr), _ptr(A.cols), _ptr(A.elms),
                               C.byref(g1), C.byref(g2), C.byref(fb)))
    if stats is not None:
        stats["fallbacks"] = fb.value
    return _csr_from_handle(g1), _csr_from_handle(g2)


def fastainv_sym_ex(A: csr_matrix, out_dtype=np.float64, row_droptol=None, row_scale=None,
                    max_elts: int = 8192000, droptol: float = 0.125, stats=None):
    """fastainv_sym with per-row drop tolerances and pivot-scale factors
    (ispm_fastainv_sym_ex).  Returns (Ainv1, Ainv2)."""
    L = _lib()
    vp = C.c_void_p
    L.ispm_fastainv_sym_ex.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, C.c_longlong,
                                       C.c_double, C.POINTER(vp), C.POINTER(vp),
                                       C.POINTER(fastainv_stats)]
    L.ispm_fastainv_sym_ex.restype = C.c_int
    odt = F64 if np.dtype(out_dtype) == np.float64 else F32
    rt = None if row_droptol is None else np.ascontiguousarray(row_droptol, np.float64)
    rs = None if row_scale is None else np.ascontiguousarray(row_scale, np.float64)
    g1, g2 = C.c_void_p(), C.c_void_p()
    st = fastainv_stats()
    _check(L.ispm_fastainv_sym_ex(odt, A.n_rows, _ptr(A.row_ptr), _ptr(A.cols), _ptr(A.elms),
                                  _ptr(rt), _ptr(rs), int(max_elts), float(droptol),
                                  C.byref(g1), C.byref(g2), C.byref(st)))
    if stats is not None:
        stats.update({k: getattr(st, k) for k, _ in fastainv_stats._fields_})
    return _csr_from_handle(g1), _csr_from_handle(g2)


# ---------------------------------------------------------------------------
# Batched PCG: many SPD systems of uneven size, 1+ right-hand sides each
# ---------------------------------------------------------------------------

_BATCH_DECLARED = False


def _declare_batch():
    global _BATCH_DECLARED
    if _BATCH_DECLARED:
        return
    _declare_solver()
    L = _lib()
    vp, i = C.c_void_p, C.c_int
    L.ispm_batch_create.argtypes = [i, vp, vp, vp, vp, vp, C.POINTER(solver_opts),
                                    C.POINTER(vp)]
    L.ispm_batch_create.restype = i
    L.ispm_batch_lanes.argtypes = [vp]
    L.ispm_batch_lanes.restype = i
    L.ispm_batch_rows.argtypes = [vp]
    L.ispm_batch_rows.restype = C.c_longlong
    L.ispm_batch_lane_info.argtypes = [vp, i, C.POINTER(i), C.POINTER(i),
                                       C.POINTER(C.c_longlong), C.POINTER(i)]
    L.ispm_batch_lane_info.restype = i
    L.ispm_batch_groups.argtypes = [vp, C.POINTER(slell_params), vp, i]
    L.ispm_batch_groups.restype = i
    L.ispm_batch_solve.argtypes = [vp, vp, vp, vp, C.POINTER(solve_stats), vp]
    L.ispm_batch_solve.restype = i
    L.ispm_batch_solve_host.argtypes = [vp, vp, vp, vp, C.POINTER(solve_stats), vp]
    L.ispm_batch_solve_host.restype = i
    L.ispm_batch_launches.argtypes = [vp]
    L.ispm_batch_launches.restype = i
    L.ispm_batch_fsai_fallbacks.argtypes = [vp]
    L.ispm_batch_fsai_fallbacks.restype = C.c_uint
    L.ispm_batch_free.argtypes = [vp]
    L.ispm_batch_free.restype = None
    _BATCH_DECLARED = True


class BatchSolver:
    """Batched PCG over independent SPD systems (ispm_batch_*).

    systems: list of FP64 csr_matrix; n_rhs: right-hand sides per system
    (int or list).  inner: np.float32 (mixed: FP32 operators and vectors,
    FP64 lane sums and reliable updates) or np.float64.  prec: "fsai_gpu" or
    "none".  Every (system, rhs) pair is a lane; lanes run together and stop
    independently."""

    def __init__(self, systems, n_rhs=1, inner=np.float32, tol: float = 1e-8,
                 max_iters: int = 100000, max_refinements: int = 500, check_every: int = 16,
                 use_graph: bool = True, prec: str = "fsai_gpu",
                 replace_ratio: float | None = None):
        _declare_batch()
        L = _lib()
        k = len(systems)
        if isinstance(n_rhs, int):
            n_rhs = [n_rhs] * k
        for A in systems:
            if A.elms.dtype != np.float64 or A.n_rows != A.n_cols:
                raise TypeError("the batched solver takes square FP64 matrices")
        o = solver_opts()
        L.ispm_solver_default_opts(C.byref(o))
        o.inner_dtype = F64 if np.dtype(inner) == np.float64 else F32
        o.tol, o.max_iters, o.max_refinements = tol, max_iters, max_refinements
        o.check_every, o.use_graph = check_every, int(use_graph)
        o.prec = {"fsai_gpu": 1, "none": 2}[prec]
        # a lane pauses for a reliable update once its recursive residual
        # fell by this factor (lanes advance in lockstep chunks)
        o.replace_ratio_f32 = 1e-3 if replace_ratio is None else replace_ratio
        if replace_ratio is not None:
            o.replace_ratio_f64 = replace_ratio
        rows = (C.c_int * k)(*[A.n_rows for A in systems])
        rhs = (C.c_int * k)(*[int(r) for r in n_rhs])
        arr = lambda f: (C.c_void_p * k)(*[_ptr(f(A)) for A in systems])
        out = C.c_void_p()
        _check(L.ispm_batch_create(k, rows, arr(lambda A: A.row_ptr), arr(lambda A: A.cols),
                                   arr(lambda A: A.elms), rhs, C.byref(o), C.byref(out)))
        self._h = out
        self.systems = list(systems)
        self.n_rhs = [int(r) for r in n_rhs]
        self.opts = o

    def __del__(self):
        if getattr(self, "_h", None) and _L is not None:
            _L.ispm_batch_free(self._h)
            self._h = None

    @property
    def lanes(self) -> int:
        return int(_lib().ispm_batch_lanes(self._h))

    @property
    def rows(self) -> int:
        return int(_lib().ispm_batch_rows(self._h))

    def lane_info(self, lane: int) -> dict:
        s, r, g = C.c_int(), C.c_int(), C.c_int()
        r0 = C.c_longlong()
        _check(_lib().ispm_batch_lane_info(self._h, lane, C.byref(s), C.byref(r), C.byref(r0),
                                           C.byref(g)))
        return {"system": s.value, "rhs": r.value, "row0": r0.value, "group": g.value}

    def groups(self):
        """[(slell_params of the group's A, lanes), ...]"""
        n = _lib().ispm_batch_groups(self._h, None, None, 0)
        fm = (slell_params * max(n, 1))()
        ln = (C.c_int * max(n, 1))()
        _lib().ispm_batch_groups(self._h, fm, ln, n)
        return [((fm[g].S, fm[g].H, fm[g].V, fm[g].D), ln[g]) for g in range(n)]

    @property
    def launches(self) -> int:
        return int(_lib().ispm_batch_launches(self._h))

    @property
    def fsai_fallbacks(self) -> int:
        return int(_lib().ispm_batch_fsai_fallbacks(self._h))

    def _finish(self, rc, lanes, tot):
        # a lane whose right-hand side holds NaN / Inf stops with ERR_INVALID
        # in its own status; the other lanes' results stand
        lane_invalid = any(lanes[l].status == ERR_INVALID for l in range(len(lanes)))
        if rc not in (OK, ERR_NOT_CONVERGED, ERR_BREAKDOWN) and not (
                rc == ERR_INVALID and lane_invalid):
            _check(rc)
        return [lanes[l].as_dict() for l in range(len(lanes))], tot.as_dict()

    def solve(self, b, x, stream=None):
        """b, x: stacked FP64 device vectors of `rows` entries.  Returns
        (per-lane stats, totals)."""
        lanes = (solve_stats * self.lanes)()
        tot = solve_stats()
        rc = _lib().ispm_batch_solve(self._h, _ptr(b), _ptr(x), lanes, C.byref(tot),
                                     _stream(stream))
        return self._finish(rc, lanes, tot)

    def solve_host(self, bs, stream=None, out=None):
        """bs[k]: system k's right-hand sides, shape (n_rhs[k], n) or (n,).
        Returns (xs, per-lane stats, totals) with xs[k] shaped like bs[k]."""
        k = len(self.systems)
        bb = [np.ascontiguousarray(b, np.float64) for b in bs]
        for j in range(k):
            if bb[j].size != self.n_rhs[j] * self.systems[j].n_rows:
                raise ValueError(f"system {j}: expected {self.n_rhs[j]} x "
                                 f"{self.systems[j].n_rows} right-hand side values")
        xs = [np.zeros_like(b) for b in bb] if out is None else out
        lanes = (solve_stats * self.lanes)()
        tot = solve_stats()
        bp = (C.c_void_p * k)(*[_ptr(b) for b in bb])
        xp = (C.c_void_p * k)(*[_ptr(x) for x in xs])
        rc = _lib().ispm_batch_solve_host(self._h, bp, xp, lanes, C.byref(tot), _stream(stream))
        st, tt = self._finish(rc, lanes, tot)
        return xs, st, tt


def shard_lpt(costs, world: int):
    """Longest-processing-time assignment of independent systems to `world`
    ranks: systems in decreasing cost order, each to the least-loaded rank
    (ties to the lowest rank).  Returns a list of system indices per rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda j: (load[j], j))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in out]
