"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes front end of the two oracle libraries:
  liboracle.so         -- the project's CPU restatement (ispm_oracle.c)
  _ref/libispm_ref.so  -- the reference's own host code compiled in place
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libispm_ref.so")

_orc = None
_ref = None


def build():
    """Compile liboracle.so, and _ref/libispm_ref.so where the reference tree exists."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def have_ref() -> bool:
    return os.path.exists(REF_SO)


class orc_slell(C.Structure):
    _fields_ = [("n_rows", C.c_int), ("n_cols", C.c_int), ("slice_height", C.c_uint),
                ("n_slices", C.c_uint), ("hblock", C.c_uint), ("var_height", C.c_int),
                ("diags", C.c_int), ("slice_ptr", C.c_void_p), ("cols", C.c_void_p),
                ("elms", C.c_void_p), ("e_f64", C.c_int)]


class ref_slell(C.Structure):
    _fields_ = [("n_rows", C.c_int), ("n_cols", C.c_int), ("n_nz", C.c_int),
                ("slice_height", C.c_uint), ("n_slices", C.c_uint), ("hblock", C.c_uint),
                ("var_height", C.c_int), ("diags", C.c_int),
                ("n_slice_ptr", C.c_longlong), ("n_cols_arr", C.c_longlong),
                ("n_elms", C.c_longlong),
                ("slice_ptr", C.c_void_p), ("cols", C.c_void_p), ("elms", C.c_void_p)]


class ref_csr(C.Structure):
    _fields_ = [("n_rows", C.c_int), ("n_cols", C.c_int), ("n_nz", C.c_int),
                ("row_ptr", C.c_void_p), ("cols", C.c_void_p), ("elms", C.c_void_p)]


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        vp, i, u, d = C.c_void_p, C.c_int, C.c_uint, C.c_double
        L.orc_slell_spmv_kernel_order.argtypes = [C.POINTER(orc_slell), u, u, i, i, vp, vp]
        L.orc_slell_spmv_exact.argtypes = [C.POINTER(orc_slell), i, i, vp, vp, vp]
        L.orc_csr_spmv_f64.argtypes = [i, vp, vp, vp, vp, vp, vp]
        L.orc_csr_spmv_f64.restype = None
        L.orc_csr_spmv_f32e.argtypes = [i, vp, vp, vp, vp, vp]
        L.orc_csr_spmv_f32e.restype = None
        L.orc_copy_indexed.argtypes = [i, vp, vp, vp, i]
        L.orc_copy_indexed.restype = None
        L.orc_add_indexed.argtypes = [i, vp, vp, vp, i]
        L.orc_add_indexed.restype = None
        L.orc_dot.argtypes = [i, vp, vp, i]
        L.orc_dot.restype = d
        L.orc_ppcg_update_scalars.argtypes = [i, vp, vp, vp, vp, vp]
        L.orc_ppcg_update_scalars.restype = None
        L.orc_ppcg_update_vectors.argtypes = [i] + [vp] * 15 + [i]
        L.orc_ppcg_update_vectors.restype = None
        L.orc_pcg_f64.argtypes = [i, i] + [vp] * 9 + [vp, vp, d, i, vp]
        L.orc_pcg_f64.restype = i
        L.orc_num_threads.restype = i
        L.orc_fsai_pattern_size.argtypes = [vp, vp, vp, i]
        L.orc_fsai_pattern_size.restype = C.c_longlong
        L.orc_fsai_rows.argtypes = [vp, vp, vp, vp, i, vp, vp, vp]
        L.orc_fsai_rows.restype = C.c_longlong
        _orc = L
    return _orc


def ref():
    global _ref
    if _ref is None:
        if not have_ref():
            build()
        if not have_ref():
            raise FileNotFoundError("oracle/_ref/libispm_ref.so is not built (reference tree absent)")
        L = C.CDLL(REF_SO)
        vp, i, d, ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
        L.ref_csr_to_slell.argtypes = [i, i, i, vp, vp, vp, i, i, i, i, i,
                                       C.POINTER(ref_slell), C.POINTER(C.c_int)]
        L.ref_csr_to_slell_guess_format.argtypes = [i, i, i, vp, vp, vp, i, i,
                                                    C.POINTER(ref_slell), C.POINTER(C.c_int)]
        L.ref_slell_free.argtypes = [C.POINTER(ref_slell)]
        L.ref_slell_free.restype = None
        L.ref_fastainv_sym.argtypes = [i, i, vp, vp, vp, ll, d, C.POINTER(ref_csr),
                                       C.POINTER(ref_csr), C.POINTER(ll)]
        L.ref_csr_free.argtypes = [C.POINTER(ref_csr)]
        L.ref_csr_free.restype = None
        L.ref_tuner_new.argtypes = [d, d]
        L.ref_tuner_new.restype = vp
        for n in ("ref_tuner_free", "ref_tuner_restart", "ref_tuner_reset_phase"):
            getattr(L, n).argtypes = [vp]
            getattr(L, n).restype = None
        for n in ("ref_tuner_get_droptol", "ref_tuner_get_best_droptol"):
            getattr(L, n).argtypes = [vp]
            getattr(L, n).restype = d
        L.ref_tuner_note_time.argtypes = [vp, d]
        L.ref_tuner_note_time.restype = None
        L.ref_tuner_iterations.argtypes = [vp]
        L.ref_tuner_iterations.restype = i
        _ref = L
    return _ref


def _np_copy(ptr, n, dt):
    if n == 0:
        return np.zeros(0, dt)
    size = n * np.dtype(dt).itemsize
    return np.frombuffer((C.c_char * size).from_address(ptr), dtype=dt, count=n).copy()


def _slell_dict(s: ref_slell, f64: bool, padded: int):
    return dict(n_rows=s.n_rows, n_cols=s.n_cols, n_nz=s.n_nz, slice_height=s.slice_height,
                n_slices=s.n_slices, hblock=s.hblock, var_height=bool(s.var_height),
                diags=bool(s.diags), padded_rows=padded,
                slice_ptr=_np_copy(s.slice_ptr, s.n_slice_ptr, np.uint32),
                cols=_np_copy(s.cols, s.n_cols_arr, np.uint32),
                elms=_np_copy(s.elms, s.n_elms, np.float64 if f64 else np.float32))


def ref_csr_to_slell(n_rows, n_cols, row_ptr, cols, elms, S, hblock, var_height, use_diags,
                     min_height=4):
    """Reference csr_to_slell (formats/conversion.h:338-414)."""
    L = ref()
    f64 = elms.dtype == np.float64
    out, padded = ref_slell(), C.c_int()
    L.ref_csr_to_slell(int(f64), n_rows, n_cols, row_ptr.ctypes.data, cols.ctypes.data,
                       elms.ctypes.data, S, hblock, int(var_height), int(use_diags), min_height,
                       C.byref(out), C.byref(padded))
    d = _slell_dict(out, f64, padded.value)
    L.ref_slell_free(C.byref(out))
    return d


def ref_csr_to_slell_guess_format(n_rows, n_cols, row_ptr, cols, elms, examine_ratio=1,
                                  min_height=4):
    """Reference csr_to_slell_guess_format (formats/conversion.h:416-492)."""
    L = ref()
    f64 = elms.dtype == np.float64
    out, padded = ref_slell(), C.c_int()
    L.ref_csr_to_slell_guess_format(int(f64), n_rows, n_cols, row_ptr.ctypes.data,
                                    cols.ctypes.data, elms.ctypes.data, examine_ratio,
                                    min_height, C.byref(out), C.byref(padded))
    d = _slell_dict(out, f64, padded.value)
    L.ref_slell_free(C.byref(out))
    return d


def ref_fastainv_sym(n, row_ptr, cols, elms, out_f64=True, max_elts=8192000, droptol=0.125):
    """Reference fastainv_sym (fastainv/fastainv.cpp:395-566).
    Returns (Ainv1, Ainv2, progress_calls) with Ainv* = (row_ptr, cols, elms)."""
    L = ref()
    a1, a2, calls = ref_csr(), ref_csr(), C.c_longlong()
    ok = L.ref_fastainv_sym(int(out_f64), n, row_ptr.ctypes.data, cols.ctypes.data,
                            elms.ctypes.data, int(max_elts), float(droptol), C.byref(a1),
                            C.byref(a2), C.byref(calls))
    if not ok:
        return None, None, calls.value
    dt = np.float64 if out_f64 else np.float32

    def take(c):
        t = (_np_copy(c.row_ptr, c.n_rows + 1, np.int32), _np_copy(c.cols, c.n_nz, np.int32),
             _np_copy(c.elms, c.n_nz, dt))
        L.ref_csr_free(C.byref(c))
        return t

    return take(a1), take(a2), calls.value


class RefDroptolTuner:
    """Reference DroptolTuner (fastainv/droptol-tuning.h:4-103)."""

    def __init__(self, lo=-10.0, hi=-3.0):
        self._L = ref()
        self._h = self._L.ref_tuner_new(lo, hi)

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.ref_tuner_free(self._h)
            self._h = None

    def getDroptol(self):
        return self._L.ref_tuner_get_droptol(self._h)

    def getBestDroptol(self):
        return self._L.ref_tuner_get_best_droptol(self._h)

    def noteTime(self, t):
        self._L.ref_tuner_note_time(self._h, float(t))

    def restart(self):
        self._L.ref_tuner_restart(self._h)

    def resetPhase(self):
        self._L.ref_tuner_reset_phase(self._h)

    def iterations(self):
        return self._L.ref_tuner_iterations(self._h)


# ---- CPU restatement front end -------------------------------------------

def _orc_struct(m: dict):
    s = orc_slell()
    s.n_rows, s.n_cols = int(m["n_rows"]), int(m["n_cols"])
    s.slice_height, s.n_slices, s.hblock = int(m["slice_height"]), int(m["n_slices"]), int(m["hblock"])
    s.var_height, s.diags = int(bool(m["var_height"])), int(bool(m["diags"]))
    keep = [np.ascontiguousarray(m["slice_ptr"], np.uint32),
            np.ascontiguousarray(m["cols"], np.uint32) if len(m["cols"]) else np.zeros(1, np.uint32),
            np.ascontiguousarray(m["elms"])]
    s.slice_ptr, s.cols, s.elms = keep[0].ctypes.data, keep[1].ctypes.data, keep[2].ctypes.data
    s.e_f64 = int(keep[2].dtype == np.float64)
    return s, keep


def slell_spmv_kernel_order(m: dict, x: np.ndarray, N: int, H: int, tex_bounds=False):
    """y = A x in the reference kernel's summation order (cuda/spmv/kernel.h)."""
    s, keep = _orc_struct(m)
    y = np.zeros(int(m["n_rows"]), x.dtype)
    rc = orc().orc_slell_spmv_kernel_order(C.byref(s), N, H, int(tex_bounds),
                                           int(x.dtype == np.float64), x.ctypes.data,
                                           y.ctypes.data)
    if rc != 0:
        raise ValueError("invalid (N, H) for this matrix")
    return y


def slell_spmv_exact(m: dict, x: np.ndarray, tex_bounds=False):
    """(y, |A||x|) accumulated in long double, following the slice walk."""
    s, keep = _orc_struct(m)
    n = int(m["n_rows"])
    y, a = np.zeros(n), np.zeros(n)
    orc().orc_slell_spmv_exact(C.byref(s), int(tex_bounds), int(x.dtype == np.float64),
                               x.ctypes.data, y.ctypes.data, a.ctypes.data)
    return y, a


def csr_spmv_f64(row_ptr, cols, elms, x):
    n = len(row_ptr) - 1
    y, a = np.zeros(n), np.zeros(n)
    if elms.dtype == np.float32:
        orc().orc_csr_spmv_f32e(n, row_ptr.ctypes.data, cols.ctypes.data, elms.ctypes.data,
                                np.ascontiguousarray(x, np.float64).ctypes.data, y.ctypes.data)
        return y
    xx = np.ascontiguousarray(x, np.float64)
    orc().orc_csr_spmv_f64(n, row_ptr.ctypes.data, cols.ctypes.data, elms.ctypes.data,
                           xx.ctypes.data, y.ctypes.data, a.ctypes.data)
    return y


def fsai_lower_f64(row_ptr, cols, elms):
    """FSAI factor on A's lower pattern (the construction the GPU build runs):
    row i solves A[P,P] y = e_i with P = {j <= i : a_ij != 0}, then
    g_i = y / sqrt(y_i).  Dense per-row solves in FP64 -- small matrices only.
    Returns (row_ptr, cols, vals) of G; rows whose local matrix is not
    positive definite become Jacobi rows."""
    n = len(row_ptr) - 1
    g_rp = [0]
    g_ci, g_v = [], []
    # dictionary of keys for symmetric lookups
    lookup = {}
    for i in range(n):
        for e in range(row_ptr[i], row_ptr[i + 1]):
            lookup[(i, int(cols[e]))] = float(elms[e])
    for i in range(n):
        P = [int(c) for c in cols[row_ptr[i]:row_ptr[i + 1]] if c <= i]
        K = len(P)
        sub = np.array([[lookup.get((P[a], P[b]), 0.0) for b in range(K)] for a in range(K)])
        try:
            Lc = np.linalg.cholesky(sub)
            e = np.zeros(K)
            e[-1] = 1.0
            y = np.linalg.solve(Lc.T, np.linalg.solve(Lc, e))
            g = y / np.sqrt(y[-1])
        except np.linalg.LinAlgError:
            g = np.zeros(K)
            aii = lookup[(i, i)]
            g[-1] = 1.0 / np.sqrt(aii) if aii > 0 else 1.0
        g_ci.extend(P)
        g_v.extend(g)
        g_rp.append(len(g_ci))
    return (np.array(g_rp, np.int32), np.array(g_ci, np.int32), np.array(g_v))


def fsai_rows_f64(row_ptr, cols, elms, rows):
    """FSAI rows (same construction as fsai_lower_f64) for the listed rows only,
    in C with OpenMP: for full-size matrices, or seeded samples of their rows.
    Returns (row_ptr, cols, vals, jacobi_rows) with row k of the result being
    row rows[k] of G."""
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(cols, np.int32)
    v = np.ascontiguousarray(elms, np.float64)
    rw = np.ascontiguousarray(rows, np.int32)
    L = orc()
    nnz = L.orc_fsai_pattern_size(rp.ctypes.data, ci.ctypes.data, rw.ctypes.data, len(rw))
    orp = np.zeros(len(rw) + 1, np.int32)
    oci = np.zeros(max(nnz, 1), np.int32)
    ov = np.zeros(max(nnz, 1), np.float64)
    jac = L.orc_fsai_rows(rp.ctypes.data, ci.ctypes.data, v.ctypes.data, rw.ctypes.data,
                          len(rw), orp.ctypes.data, oci.ctypes.data, ov.ctypes.data)
    if jac < 0:
        raise ValueError("an FSAI row pattern is empty or exceeds 64 entries")
    return orp, oci[:nnz], ov[:nnz], int(jac)


def pcg_f64(A, b, G1=None, G2=None, pipelined=False, tol=1e-10, max_it=100000, x0=None):
    """FP64 PCG on CSR triples (row_ptr, cols, elms); returns (x, iters, relres)."""
    n = len(A[0]) - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    rel = C.c_double()
    g1 = G1 if G1 is not None else (None, None, None)
    g2 = G2 if G2 is not None else (None, None, None)

    def p(a):
        return None if a is None else np.ascontiguousarray(a).ctypes.data

    it = orc().orc_pcg_f64(int(pipelined), n, p(A[0]), p(A[1]), p(A[2]), p(g1[0]), p(g1[1]),
                           p(g1[2]), p(g2[0]), p(g2[1]), p(g2[2]),
                           np.ascontiguousarray(b, np.float64).ctypes.data, x.ctypes.data,
                           float(tol), int(max_it), C.byref(rel))
    return x, it, rel.value
