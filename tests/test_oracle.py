"""Pins of the CPU oracle itself (no GPU).

The reference's kernels cannot be compiled with CUDA 12, so the SpMV oracle
is a restatement of cuda/spmv/kernel.h.  It is pinned here by properties that
hold for any correct walk of the layout: on matrices converted by the
reference's own conversion code (oracle/_ref), the slice walk must reproduce
the CSR product, in both the exact and the reference-summation-order modes,
for every format and launch shape."""
import numpy as np
import pytest

from conftest import copy_csr

MODES = [(32, 1, 0, 1), (64, 1, 0, 0), (32, 2, 0, 0), (64, 4, 0, 0), (256, 1, 1, 0),
         (256, 1, 1, 1), (128, 2, 1, 0), (16, 1, 0, 1)]


def _ref_slell(ref, A, mode):
    S, W, V, D = mode
    return ref.ref_csr_to_slell(A.n_rows, A.n_cols, A.row_ptr, A.cols, A.elms, S, W, V, D)


@pytest.mark.parametrize("mode", MODES)
def test_oracle_walk_reproduces_csr_product(ref, gen, mode):
    for A in (gen.poisson7(10), gen.random_csr(1200, 1200, 3, mean_len=9, band=30),
              gen.random_csr(500, 1100, 4, mean_len=12, pair_frac=0.6),
              gen.unstructured(8, seed=2)):
        m = _ref_slell(ref, A, mode)
        x = np.random.default_rng(0).uniform(-1, 1, A.n_cols)
        y_csr = ref.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x)
        y, absrow = ref.slell_spmv_exact(m, x)
        assert np.all(y[A.n_rows:] == 0)
        assert np.allclose(y[: A.n_rows], y_csr, rtol=0, atol=1e-13 * max(1, absrow.max()))
        for N, H in ((64, 1), (256, 2), (512, 1), (128, 4)):
            sz = m["slice_height"] if not m["var_height"] else N * H
            try:
                yk = ref.slell_spmv_kernel_order(m, x, N, H)
            except ValueError:
                continue
            assert np.allclose(yk[: A.n_rows], y_csr, rtol=0,
                               atol=1e-13 * max(1, absrow.max())), (N, H, sz)


def test_texture_bound_quirk_is_confined(ref, gen):
    """With hblock 2 and odd n_cols the reference's W-wide x texture covers
    floor(n_cols / 2) vectors (cuda/spmv/dispatch.h:46-49): a single at column
    n_cols - 1 spilled into a block slot reads 0.  The product bounds each
    element instead; the two agree everywhere except on such rows."""
    A = gen.random_csr(1001, 1001, 42, mean_len=7, pair_frac=0.9)
    m = _ref_slell(ref, A, (32, 2, 0, 0))
    x = np.random.default_rng(1).uniform(-1, 1, A.n_cols)
    y_exact, _ = ref.slell_spmv_exact(m, x, tex_bounds=False)
    y_tex, _ = ref.slell_spmv_exact(m, x, tex_bounds=True)
    y_csr = ref.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x)
    assert np.allclose(y_exact[: A.n_rows], y_csr, atol=1e-12)
    diff = np.nonzero(np.abs(y_tex[: A.n_rows] - y_csr) > 1e-12)[0]
    # every differing row holds an entry in the last column
    last = A.n_cols - 1
    for r in diff:
        assert last in A.cols[A.row_ptr[r]:A.row_ptr[r + 1]]


def test_oracle_sblas_recurrences(oracle):
    rng = np.random.default_rng(3)
    n = 1000
    vec = {k: rng.standard_normal(n) for k in "nmpsqzxruw"}
    a, b = np.array([0.7]), np.array([0.3])
    v = {k: vec[k].copy() for k in vec}
    red = np.zeros(3)
    oracle.orc().orc_ppcg_update_vectors(1, red[0:].ctypes.data, red[1:].ctypes.data,
                                         red[2:].ctypes.data,
                                         a.ctypes.data, b.ctypes.data, v["n"].ctypes.data,
                                         v["m"].ctypes.data, *[v[k].ctypes.data for k in "psqzxruw"],
                                         n)
    z = vec["n"] + 0.3 * vec["z"]
    q = vec["m"] + 0.3 * vec["q"]
    s = vec["w"] + 0.3 * vec["s"]
    p = vec["u"] + 0.3 * vec["p"]
    u = vec["u"] - 0.7 * q
    w = vec["w"] - 0.7 * z
    r = vec["r"] - 0.7 * s
    x = vec["x"] + 0.7 * p
    for k, ref_v in zip("zqspuwrx", (z, q, s, p, u, w, r, x)):
        assert np.allclose(v[k], ref_v, rtol=1e-15, atol=1e-15)
    assert np.isclose(red[0], np.abs(r).sum(), rtol=1e-14)
    assert np.isclose(red[1], r @ u, rtol=1e-12)
    assert np.isclose(red[2], w @ u, rtol=1e-12)


def test_oracle_pcg_converges_c1(ref, gen, ispm):
    """Config 1 on the CPU: 32^3 Poisson, FSAI droptol 0.01 from the
    reference's own fastainv, classic and pipelined PCG to 1e-8."""
    A = gen.poisson7(32)
    x_true = np.random.default_rng(0).uniform(-1, 1, A.n_rows)
    b = ref.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x_true)
    g1, g2, _ = ref.ref_fastainv_sym(A.n_rows, A.row_ptr, A.cols, A.elms, True, 8192000, 0.01)
    Acsr = (A.row_ptr, A.cols, A.elms)
    its = {}
    for pipe in (False, True):
        x, it, rel = ref.pcg_f64(Acsr, b, g1, g2, pipelined=pipe, tol=1e-8)
        assert rel <= 1.5e-8
        its[pipe] = it
    x0, it0, _ = ref.pcg_f64(Acsr, b, None, None, tol=1e-8)
    assert abs(its[True] - its[False]) <= 2
    assert its[False] < it0  # the preconditioner pays
