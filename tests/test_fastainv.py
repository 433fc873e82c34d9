"""fastainv_sym: bit-exact against the reference (fastainv/fastainv.cpp:395-566)
through the golden fixtures and, where oracle/_ref is built, live."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

_Z = np.load(os.path.join(GOLDEN, "fastainv.npz"))
_CASES = sorted({k.split("/")[0] for k in _Z.files})


def _bits_equal(a, b):
    return a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("name", _CASES)
def test_fastainv_matches_golden(ispm, name):
    z = _Z
    f64, max_elts, droptol, calls = z[f"{name}/params"]
    rp, ci, el = z[f"{name}/A_row_ptr"], z[f"{name}/A_cols"], z[f"{name}/A_elms"]
    A = ispm.csr_matrix(len(rp) - 1, len(rp) - 1, rp, ci, el)
    count = [0]
    g1, g2 = ispm.fastainv_sym(A, np.float64 if f64 else np.float32,
                               lambda: count.__setitem__(0, count[0] + 1), int(max_elts),
                               float(droptol))
    assert count[0] == int(calls)  # progress once per row, as the reference
    for tag, g in (("G1", g1), ("G2", g2)):
        assert np.array_equal(g.row_ptr, z[f"{name}/{tag}_row_ptr"])
        assert np.array_equal(g.cols, z[f"{name}/{tag}_cols"])
        assert _bits_equal(g.elms, z[f"{name}/{tag}_elms"])


def _live(gen):
    return [
        ("poisson7_16_dt0.01", gen.poisson7(16), 8192000, 0.01),
        ("grf27_12_dt0.01", gen.stencil_grf(12, 27, 4.0, 1.5, 7), 50_000_000, 0.01),
        ("grf7_14_dt0.003", gen.stencil_grf(14, 7, 4.0, 2.0, 8), 50_000_000, 0.003),
        ("unstr12_dt0.02", gen.unstructured(12, seed=9), 50_000_000, 0.02),
        ("grf27_10_trunc", gen.stencil_grf(10, 27, 3.0, 1.5, 6), 30_000, 0.002),
        ("poisson7_10_dt0", gen.poisson7(10), 50_000_000, 0.0),
        ("poisson7_12_dt1", gen.poisson7(12), 8192000, 1.0),
    ]


@pytest.mark.parametrize("f64", [True, False])
def test_fastainv_matches_reference_live(ispm, ref, gen, f64):
    for name, A, max_elts, dt in _live(gen):
        r1, r2, calls = ref.ref_fastainv_sym(A.n_rows, A.row_ptr, A.cols, A.elms, f64,
                                             max_elts, dt)
        st = {}
        g1, g2 = ispm.fastainv_sym(A, np.float64 if f64 else np.float32, None, max_elts, dt,
                                   stats=st)
        for g, r in ((g1, r1), (g2, r2)):
            assert np.array_equal(g.row_ptr, r[0]), name
            assert np.array_equal(g.cols, r[1]), name
            assert _bits_equal(g.elms, r[2]), name
        if "trunc" in name:
            assert st["truncated_rows"] > 0 and st["chunks_used"] == st["storage_chunks"]


def test_fastainv_breakdown_and_indefinite(ispm, ref):
    # A symmetric matrix with a zero pivot (row 1 has D_11 = 0 after row 0) and
    # a negative pivot: the signed / unsigned scale split of Ainv1 / Ainv2
    # (fastainv.cpp:518-519) and the breakdown path (fastainv.cpp:468-472).
    n = 6
    dense = np.array([[2, 2, 0, 0, 0, 0],
                      [2, 2, 1, 0, 0, 0],
                      [0, 1, -3, 1, 0, 0],
                      [0, 0, 1, 4, 1, 0],
                      [0, 0, 0, 1, -5, 2],
                      [0, 0, 0, 0, 2, 6]], np.float64)
    rows, cols = np.nonzero(dense)
    rp = np.zeros(n + 1, np.int32)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    A = ispm.csr_matrix(n, n, rp, cols.astype(np.int32), dense[rows, cols])
    st = {}
    g1, g2 = ispm.fastainv_sym(A, np.float64, None, 8192000, 0.0, stats=st)
    r1, r2, _ = ref.ref_fastainv_sym(n, A.row_ptr, A.cols, A.elms, True, 8192000, 0.0)
    assert st["breakdowns"] >= 1
    assert _bits_equal(g1.elms, r1[2]) and _bits_equal(g2.elms, r2[2])
    assert np.array_equal(g1.cols, r1[1]) and np.array_equal(g2.cols, r2[1])


def test_preconditioner_is_an_approximate_inverse(ispm, gen):
    # M = Ainv2 Ainv1 ~ A^-1: with droptol 0 on a small SPD matrix, exact.
    A = gen.stencil_grf(5, 7, 2.0, 1.0, 1)
    g1, g2 = ispm.fastainv_sym(A, np.float64, None, 50_000_000, 0.0)
    Ad = A.to_scipy().toarray()
    M = g2.to_scipy().toarray() @ g1.to_scipy().toarray()
    assert np.allclose(M @ Ad, np.eye(A.n_rows), atol=1e-9)
