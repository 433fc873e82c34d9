"""GPU FSAI build: a parallel replacement for the reference's serial host
build of the approximate inverse (fastainv/fastainv.cpp:395-566), judged
residual-equivalent: its factor matches the CPU FSAI oracle (same
construction, dense per-row solves in FP64) to rounding, and PCG with it
converges to the same true residual in about the AINV iteration count."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["poisson7_10", "grf27_9", "grf7_12", "unstructured_8"])
def test_fsai_values_match_oracle(ispm, oracle, cuda, gen, name):
    A = {"poisson7_10": lambda: gen.poisson7(10),
         "grf27_9": lambda: gen.stencil_grf(9, 27, 3.0, 1.5, 4),
         "grf7_12": lambda: gen.stencil_grf(12, 7, 4.0, 2.0, 5),
         "unstructured_8": lambda: gen.unstructured(8, seed=6)}[name]()
    st = {}
    G1, G2 = ispm.fsai_sym_gpu(A, np.float64, stats=st)
    rp, ci, v = oracle.fsai_lower_f64(A.row_ptr, A.cols, A.elms)
    assert st["fallbacks"] == 0
    assert np.array_equal(G1.row_ptr, rp) and np.array_equal(G1.cols, ci)
    assert np.allclose(G1.elms, v, rtol=1e-11, atol=1e-13 * np.abs(v).max())
    # Ainv2 = G^T exactly (same values, transposed)
    assert np.array_equal(G2.to_scipy().toarray(), G1.to_scipy().toarray().T)
    # FSAI normalisation: diag(G A G^T) = 1
    Gs, As = G1.to_scipy(), A.to_scipy()
    assert np.allclose((Gs @ As @ Gs.T).diagonal(), 1.0, atol=1e-10)


def test_fsai_fp32_output_and_fallback(ispm, cuda):
    # a matrix with one non-positive-definite local block: row 2's local
    # matrix [[1, 3], [3, 1]] is indefinite -> Jacobi row
    dense = np.array([[4., 0, 0, 0], [0, 1, 3, 0], [0, 3, 1, 0], [0, 0, 0, 2]])
    rows, cols = np.nonzero(dense)
    rp = np.zeros(5, np.int32)
    np.add.at(rp, rows + 1, 1)
    A = ispm.csr_matrix(4, 4, np.cumsum(rp).astype(np.int32), cols.astype(np.int32),
                        dense[rows, cols])
    st = {}
    G1, G2 = ispm.fsai_sym_gpu(A, np.float32, stats=st)
    assert G1.elms.dtype == np.float32 and st["fallbacks"] == 1
    g = G1.to_scipy().toarray()
    assert g[2, 1] == 0 and np.isclose(g[2, 2], 1.0)  # Jacobi row for a_22 = 1
    assert np.isclose(g[0, 0], 0.5) and np.isclose(g[3, 3], 1 / np.sqrt(2))


def test_pcg_with_gpu_fsai(ispm, oracle, cuda, gen):
    A = gen.stencil_grf(32, 27, 8.0, 1.5, 0)
    x_true = np.random.default_rng(0).uniform(-1, 1, A.n_rows)
    b = oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x_true)
    G1, G2 = ispm.fastainv_sym(A, np.float64, None, 200_000_000, 0.01)
    its = {}
    # fsai_gpu32: the internal build with FP32 factor values, the operator the
    # exported pair gives (the default stores an FP32 inner solve's factor
    # as FP16 x 2^k, a slightly different preconditioner)
    for label, kw in (("ainv", dict(G1=G1, G2=G2)), ("fsai_gpu", dict(prec="fsai_gpu")),
                      ("fsai_gpu32", dict(prec="fsai_gpu", factor_f16=False)),
                      ("fsai_pair", "pair")):
        if kw == "pair":
            F1, F2 = ispm.fsai_sym_gpu(A, np.float64)
            kw = dict(G1=F1, G2=F2)
        for inner in (np.float64, np.float32):
            s = ispm.PCGSolver(A, inner=inner, tol=1e-10, **kw)
            x, st = s.solve_host(b)
            assert st["converged"], (label, st)
            r = b - oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x)
            assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10 * 1.001
            its[(label, inner)] = st["iterations"]
    # residual-equivalent: within 15% of the AINV iteration count
    for inner in (np.float64, np.float32):
        assert its[("fsai_gpu", inner)] <= 1.15 * its[("ainv", inner)], its
        assert its[("fsai_gpu32", inner)] == its[("fsai_pair", inner)], its
        assert abs(its[("fsai_gpu", inner)] - its[("fsai_pair", inner)]) <= 3, its


@pytest.mark.parametrize("prec", ["fsai_gpu", "ainv"])
def test_bf16_factor_values(ispm, oracle, cuda, gen, prec):
    """Mixed solve with the factor's values kept in BF16 (half the bytes of
    each factor application): it meets the same true-residual target, in at
    most 10% more iterations than with FP32 factor values."""
    A = gen.stencil_grf(24, 27, 8.0, 1.5, 0)
    b = oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms,
                            np.random.default_rng(0).uniform(-1, 1, A.n_rows))
    kw = dict(prec="fsai_gpu")
    if prec == "ainv":
        G1, G2 = ispm.fastainv_sym(A, np.float64, None, 200_000_000, 0.01)
        kw = dict(G1=G1, G2=G2)
    its = {}
    for bf in (False, True):
        S = ispm.PCGSolver(A, inner=np.float32, tol=1e-10, factor_bf16=bf, **kw)
        x, st = S.solve_host(b)
        assert st["converged"], st
        r = b - oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x)
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10 * 1.001
        its[bf] = st["iterations"]
    assert its[True] <= 1.1 * its[False] + 3, its


@pytest.mark.parametrize("L", [24, 48])
def test_f16_factor_values(ispm, oracle, cuda, gen, L):
    """Mixed solve with the GPU FSAI factor's values kept in FP16 times one
    power-of-two scale (half the bytes of each factor application, 11
    mantissa bits): the same true-residual target in at most 5% more
    iterations than with FP32 factor values (measured on the B200 at 128^3:
    499 against 501)."""
    A = gen.stencil_grf(L, 27, 8.0, 1.5, 0)
    b = oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms,
                            np.random.default_rng(0).uniform(-1, 1, A.n_rows))
    its = {}
    for f16 in (False, True):
        S = ispm.PCGSolver(A, inner=np.float32, tol=1e-10, prec="fsai_gpu", factor_f16=f16)
        x, st = S.solve_host(b)
        assert st["converged"], st
        r = b - oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x)
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10 * 1.001
        its[f16] = st["iterations"]
    assert its[True] <= 1.05 * its[False] + 2, its
