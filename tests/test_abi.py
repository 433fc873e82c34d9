"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import PKG, ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(ispm_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert len(names) > 40
    assert "ispm_launch_spmv" in names and "ispm_fastainv_sym" in names


def test_library_exports_all_declared_symbols(ispm):
    lib = ctypes.CDLL(os.path.join(PKG, "libispm_b200.so"))
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_error_strings_and_version(ispm):
    L = ispm.lib_handle()
    assert L.ispm_error_string(0) == b"ok"
    assert L.ispm_error_string(1) == b"invalid argument"
    assert b"sm_100a" in L.ispm_version()


def test_launch_params_valid_matches_reference_macro(ispm):
    # SPMV_PARAMS_VALID_P(N, S, H) = N >= S / H && S >= H (kernel-iface.h:4)
    for N in (64, 128, 256, 512):
        for S in (16, 32, 64, 128, 256, 512, 1024):
            for H in (1, 2):
                p = ispm.spmv_launch_params(N, S, H, 1, 1)
                assert p.valid() == (N >= S // H and S >= H)


def test_invalid_arguments_raise(ispm, gen):
    A = gen.poisson7(4)
    import pytest
    with pytest.raises(ispm.IspmError) as e:
        ispm.csr_to_slell(A, 48, 1, False, False)  # not a power of two
    assert e.value.status == ispm.ERR_INVALID
    with pytest.raises(ispm.IspmError):
        ispm.csr_to_slell(A, 32, 3, False, False)  # hblock 3
    bad = ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr, A.cols.copy(), A.elms)
    bad.cols[5] = A.n_cols + 7
    with pytest.raises(ispm.IspmError):
        ispm.csr_to_slell(bad, 32, 1, False, True)
    with pytest.raises(ispm.IspmError):
        ispm.fastainv_sym(ispm.csr_matrix(0, 0, [0], [], []))


def test_solver_default_options(ispm):
    """ispm_solver_default_opts fills the values the header documents (no GPU
    needed: it only writes the struct)."""
    import ctypes as C
    L = ispm.lib_handle()
    L.ispm_solver_default_opts.argtypes = [C.POINTER(ispm.solver_opts)]
    L.ispm_solver_default_opts.restype = None
    o = ispm.solver_opts()
    L.ispm_solver_default_opts(C.byref(o))
    assert o.inner_dtype == ispm.F32 and o.tol == 1e-10
    assert (o.max_iters, o.max_refinements, o.check_every, o.use_graph) == (100000, 500, 16, 1)
    assert o.replace_ratio_f32 == 1e-2 and o.replace_ratio_f64 == 1e-4
    assert (o.variant, o.prec, o.factor_bf16, o.reorder) == (0, 0, 0, 2)
    assert o.matrix_f16 == 0 and o.factor_f16 == 1 and o.refresh == 0


def test_solver_rejects_malformed_csr_before_reordering(ispm, gen):
    """ispm_solver_create and ispm_batch_create validate row_ptr and the column
    indices before the reverse Cuthill-McKee ordering or any conversion walks
    them (an out-of-range column used to index the ordering's work arrays).
    No GPU needed: the check comes before any device work."""
    import pytest
    A = gen.poisson7(6)
    cases = []
    bad_col = A.cols.copy()
    bad_col[7] = A.n_cols + 1000
    cases.append(("column past n", A.row_ptr, bad_col))
    neg_col = A.cols.copy()
    neg_col[11] = -5
    cases.append(("negative column", A.row_ptr, neg_col))
    bad_rp = A.row_ptr.copy()
    bad_rp[10], bad_rp[11] = bad_rp[11] + 3, bad_rp[10]
    cases.append(("decreasing row_ptr", bad_rp, A.cols))
    off_rp = A.row_ptr.copy() + 1
    cases.append(("row_ptr[0] != 0", off_rp, A.cols))
    for name, rp, ci in cases:
        M = ispm.csr_matrix(A.n_rows, A.n_cols, rp, ci, A.elms)
        for reorder in ("auto", "rcm", "none"):
            with pytest.raises(ispm.IspmError) as e:
                ispm.PCGSolver(M, inner=np.float64, prec="fsai_gpu", reorder=reorder)
            assert e.value.status == ispm.ERR_INVALID, (name, reorder)
        with pytest.raises(ispm.IspmError) as e:
            ispm.BatchSolver([A, M], 1)
        assert e.value.status == ispm.ERR_INVALID, name
    # a malformed factor pair is refused the same way
    with pytest.raises(ispm.IspmError) as e:
        ispm.PCGSolver(A, ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr, bad_col, A.elms), A,
                       inner=np.float64)
    assert e.value.status == ispm.ERR_INVALID


def test_rcm_order_is_a_permutation_that_narrows_the_band(ispm, gen):
    """ispm_rcm_order on a randomly numbered mesh: perm is a permutation and
    the renumbered matrix's bandwidth is far below the scattered one's;
    malformed patterns are refused."""
    A = gen.unstructured(12, 0.05, 3, 0.1, 10.0, 1.01)
    perm = ispm.rcm_order(A)
    assert np.array_equal(np.sort(perm), np.arange(A.n_rows))
    B = ispm.permute_symmetric(A, perm)
    assert B.row_ptr[-1] == A.row_ptr[-1]
    assert ispm.csr_bandwidth(B) * 4 <= ispm.csr_bandwidth(A)
    # P A P^T holds the same entries: (B x)[i] = (A x_perm)[perm[i]]
    x = np.random.default_rng(1).uniform(-1, 1, A.n_rows)
    import scipy.sparse as sp
    MA = sp.csr_matrix((A.elms, A.cols, A.row_ptr), shape=(A.n_rows, A.n_rows))
    MB = sp.csr_matrix((B.elms, B.cols, B.row_ptr), shape=(A.n_rows, A.n_rows))
    xa = np.empty_like(x)
    xa[perm] = x
    assert np.allclose(MB @ x, (MA @ xa)[perm], rtol=1e-14, atol=1e-14)
    bad = ispm.csr_matrix(3, 3, np.array([0, 1, 2, 3], np.int32), np.array([0, 5, 2], np.int32),
                          np.ones(3))
    with pytest.raises(ispm.IspmError):
        ispm.rcm_order(bad)
    with pytest.raises(ispm.IspmError):
        ispm.csr_bandwidth(bad)


def test_solver_shape(ispm, gen):
    """ispm_solver_choose_shape: a shape the conversion accepts, and on a
    27-point grid the 128-row diagonal-block shape (fewest bytes there)."""
    A = gen.stencil_grf(24, 27, 4.0, 1.5, 1)
    s = ispm.solver_shape(A)
    assert s == (128, 1, 0, 1)
    U = gen.unstructured(10, 0.05, 3, 0.1, 10.0, 1.01)
    S, H, V, D = ispm.solver_shape(U, np.float64)
    ispm.csr_to_slell(U, S, H, V, D)  # accepted
    bad = ispm.csr_matrix(3, 3, np.array([0, 1, 2, 3], np.int32), np.array([0, 5, 2], np.int32),
                          np.ones(3))
    with pytest.raises(ispm.IspmError):
        ispm.solver_shape(bad)
