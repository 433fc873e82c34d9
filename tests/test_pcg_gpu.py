"""Pipelined PCG on the GPU: every solve is judged by its true residual
||b - A x||_2 / ||b||_2 computed on the CPU with the FP64 CSR oracle; the
iteration counts of the FP64 path track the CPU oracle's pipelined PCG (the
sblas.cu:156-216 recurrences in FP64) on the same FSAI preconditioner."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1(ispm, gen, oracle):
    """Config 1: 32^3 7-point Poisson, x_true ~ U(-1, 1) seed 0, b = A x_true,
    FSAI droptol 0.01."""
    A = gen.poisson7(32)
    x_true = np.random.default_rng(0).uniform(-1, 1, A.n_rows)
    b = oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x_true)
    G1, G2 = ispm.fastainv_sym(A, np.float64, None, 8192000, 0.01)
    return A, b, G1, G2


def true_relres(oracle, A, b, x):
    r = b - oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x)
    return np.linalg.norm(r) / np.linalg.norm(b)


@pytest.mark.parametrize("inner", [np.float64, np.float32], ids=["fp64", "mixed"])
@pytest.mark.parametrize("tol", [1e-8, 1e-10])
def test_pcg_c1_true_residual(ispm, oracle, cuda, c1, inner, tol):
    A, b, G1, G2 = c1
    s = ispm.PCGSolver(A, G1, G2, inner=inner, tol=tol)
    x, st = s.solve_host(b)
    assert st["converged"] and st["status"] == 0, st
    rel = true_relres(oracle, A, b, x)
    assert rel <= tol * 1.001, (rel, st)
    assert abs(rel - st["true_relres"]) <= 0.05 * rel + 1e-16  # GPU FP64 residual agrees
    if inner == np.float64:
        _, it_cpu, _ = oracle.pcg_f64((A.row_ptr, A.cols, A.elms), b,
                                      (G1.row_ptr, G1.cols, G1.elms),
                                      (G2.row_ptr, G2.cols, G2.elms), pipelined=True, tol=tol)
        assert abs(st["iterations"] - it_cpu) <= max(3, 0.05 * it_cpu), (st, it_cpu)


@pytest.mark.parametrize("inner,variant", [(np.float64, "classic"), (np.float32, "pipelined")])
def test_pcg_other_variants(ispm, oracle, cuda, c1, inner, variant):
    """Classic PCG in FP64 and pipelined PCG in FP32 (with reliable updates)
    on config 1 also reach 1e-10 in the true residual."""
    A, b, G1, G2 = c1
    s = ispm.PCGSolver(A, G1, G2, inner=inner, tol=1e-10, variant=variant)
    x, st = s.solve_host(b)
    assert st["converged"], st
    assert true_relres(oracle, A, b, x) <= 1e-10 * 1.001


def test_pcg_mixed_matches_fp64_iterations(ispm, oracle, cuda, gen):
    """FP32 classic PCG with FP64 reliable updates needs about the FP64
    iteration count on a 27-point GRF system (kappa ~ 1e6)."""
    A = gen.stencil_grf(32, 27, 8.0, 1.5, 0)
    x_true = np.random.default_rng(0).uniform(-1, 1, A.n_rows)
    b = oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x_true)
    G1, G2 = ispm.fastainv_sym(A, np.float64, None, 200_000_000, 0.01)
    its = {}
    for inner in (np.float64, np.float32):
        x, st = ispm.PCGSolver(A, G1, G2, inner=inner, tol=1e-10).solve_host(b)
        assert st["converged"], st
        assert true_relres(oracle, A, b, x) <= 1e-10 * 1.001
        its[inner] = st["iterations"]
    assert its[np.float32] <= 1.1 * its[np.float64] + 5, its


def test_pcg_device_vectors_graph_and_eager_agree(ispm, oracle, cuda, c1):
    A, b, G1, G2 = c1
    outs = []
    # use_graph 2: the chunk repeats inside the graph's while node
    for use_graph in (True, False, 2):
        s = ispm.PCGSolver(A, G1, G2, inner=np.float32, tol=1e-10, use_graph=use_graph)
        bd = cuda.zeros(s.rows, dtype=cuda.float64, device="cuda")
        bd[: A.n_rows] = cuda.from_numpy(b).cuda()
        xd = cuda.zeros_like(bd)
        st = s.solve(bd, xd)
        assert st["converged"]
        outs.append((xd.cpu().numpy(), st))
    for k in (1, 2):
        assert np.array_equal(outs[0][0], outs[k][0])
        assert outs[0][1]["iterations"] == outs[k][1]["iterations"]
        assert outs[0][1]["refinements"] == outs[k][1]["refinements"]
    assert true_relres(oracle, A, b, outs[0][0][: A.n_rows]) <= 1e-10


def test_pcg_device_loop_stops(ispm, oracle, cuda, c1):
    """The while-node loop ends on every flag the direction kernel or the
    update raises: convergence without a preconditioner (the update's stop
    test), the iteration cap, and a breakdown."""
    A, b, G1, G2 = c1
    for prec in ((G1, G2), (None, None)):
        x, st = ispm.PCGSolver(A, *prec, inner=np.float32, tol=1e-9, use_graph=2,
                               check_every=4).solve_host(b)
        ref, st_ref = ispm.PCGSolver(A, *prec, inner=np.float32, tol=1e-9).solve_host(b)
        assert st["converged"] and st["iterations"] == st_ref["iterations"]
        assert np.array_equal(x, ref)
    s = ispm.PCGSolver(A, G1, G2, inner=np.float32, tol=1e-14, max_iters=5, use_graph=2)
    x, st = s.solve_host(b)
    assert not st["converged"] and st["status"] == ispm.ERR_NOT_CONVERGED
    assert st["iterations"] <= 5 + 16
    n = 64
    d = np.where(np.arange(n) % 2 == 0, 2.0, -2.0)
    rp = np.arange(n + 1, dtype=np.int32)
    Ai = ispm.csr_matrix(n, n, rp, np.arange(n, dtype=np.int32), d)
    x, st = ispm.PCGSolver(Ai, None, None, inner=np.float32, tol=1e-10, max_refinements=5,
                           use_graph=2).solve_host(np.ones(n))
    assert st["status"] == ispm.ERR_BREAKDOWN and np.all(np.isfinite(x))


def test_pcg_without_preconditioner_and_grf(ispm, oracle, cuda, gen):
    A = gen.stencil_grf(16, 27, 4.0, 1.5, 3)
    x_true = np.random.default_rng(1).uniform(-1, 1, A.n_rows)
    b = oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x_true)
    for inner in (np.float64, np.float32):
        s = ispm.PCGSolver(A, None, None, inner=inner, tol=1e-9)
        x, st = s.solve_host(b)
        assert st["converged"], st
        assert true_relres(oracle, A, b, x) <= 1e-9 * 1.001
    G1, G2 = ispm.fastainv_sym(A, np.float64, None, 50_000_000, 0.01)
    s = ispm.PCGSolver(A, G1, G2, inner=np.float32, tol=1e-10)
    x, st = s.solve_host(b)
    assert st["converged"] and true_relres(oracle, A, b, x) <= 1e-10 * 1.001


def test_pcg_zero_rhs_and_limits(ispm, oracle, cuda, c1):
    A, b, G1, G2 = c1
    s = ispm.PCGSolver(A, G1, G2, inner=np.float64, tol=1e-10)
    x, st = s.solve_host(np.zeros_like(b))
    assert st["converged"] and np.all(x == 0)
    s2 = ispm.PCGSolver(A, G1, G2, inner=np.float64, tol=1e-14, max_iters=5)
    x, st = s2.solve_host(b)
    assert not st["converged"] and st["status"] == ispm.ERR_NOT_CONVERGED
    assert st["iterations"] <= 5 + 16


def test_pcg_indefinite_matrix_stops(ispm, cuda):
    # symmetric indefinite: CG breaks down; the solver must stop and report it
    n = 64
    d = np.where(np.arange(n) % 2 == 0, 2.0, -2.0)
    rp = np.arange(n + 1, dtype=np.int32)
    A = ispm.csr_matrix(n, n, rp, np.arange(n, dtype=np.int32), d)
    # p.Ap = sum(d) = 0 on the first step: alpha is infinite, the step is
    # refused, and after three restarts that do not lower the residual the
    # solver stops with ERR_BREAKDOWN
    for inner in (np.float64, np.float32):
        s = ispm.PCGSolver(A, None, None, inner=inner, tol=1e-10, max_refinements=5)
        x, st = s.solve_host(np.ones(n))
        assert not st["converged"], (inner, st)
        assert st["status"] == ispm.ERR_BREAKDOWN, (inner, st)
        assert np.all(np.isfinite(x)) and st["true_relres"] >= 1e-10


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
@pytest.mark.parametrize("inner", [np.float32, np.float64])
def test_pcg_non_finite_rhs_is_refused(ispm, oracle, cuda, c1, bad, inner):
    """A NaN or infinite entry in b cannot be solved to a relative target: the
    solve returns ERR_INVALID at once (it used to report convergence with
    x = 0, since ||b|| compared as not positive), and the solver stays usable."""
    A, b, G1, G2 = c1
    s = ispm.PCGSolver(A, G1, G2, inner=inner, tol=1e-10)
    bb = b.copy()
    bb[123] = bad
    with pytest.raises(ispm.IspmError) as e:
        s.solve_host(bb)
    assert e.value.status == ispm.ERR_INVALID
    x, st = s.solve_host(b)
    assert st["converged"]
    r = b - oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x)
    assert np.linalg.norm(r) <= 1.001e-10 * np.linalg.norm(b)


@pytest.mark.parametrize("inner", [np.float32, np.float64])
def test_reordered_solve_of_a_permuted_mesh(ispm, oracle, cuda, gen, inner):
    """A randomly numbered mesh solved with and without the solver's reverse
    Cuthill-McKee renumbering: b and x stay in the caller's order, every
    solve meets the tolerance against the FP64 CSR oracle, and the solutions
    agree."""
    A = gen.unstructured(20, 0.05, 3, 0.1, 10.0, 1.01)
    x_true = np.random.default_rng(5).uniform(-1, 1, A.n_rows)
    b = oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x_true)
    xs = {}
    for mode in ("none", "rcm", "auto"):
        S = ispm.PCGSolver(A, inner=inner, tol=1e-10, prec="fsai_gpu", reorder=mode)
        x, st = S.solve_host(b)
        assert st["converged"], (mode, st)
        r = b - oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x)
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10 * 1.001, mode
        xs[mode] = x
    for mode in ("rcm", "auto"):
        assert np.allclose(xs[mode], xs["none"], rtol=0, atol=1e-7 * np.abs(x_true).max())


def test_reordering_rejects_a_given_pair(ispm, cuda, gen):
    A = gen.poisson7(6)
    G1, G2 = ispm.fastainv_sym(A, np.float64, None, 8_000_000, 0.01)
    with pytest.raises(ispm.IspmError):
        ispm.PCGSolver(A, G1, G2, reorder="rcm")
    ispm.PCGSolver(A, G1, G2, reorder="auto")  # automatic mode leaves it alone


@pytest.mark.parametrize("inner,f16", [(np.float32, False), (np.float64, False),
                                       (np.float32, True)], ids=["f32", "f64", "f32-split"])
def test_solver_edge_cases(ispm, oracle, cuda, gen, inner, f16):
    """Zero right-hand side (x = 0 at once), a 1 x 1 system and a system the
    starting guess already solves exactly; also with A's inner copy stored as
    the FP16 split (f32-split), where the 1 x 1 and diagonal systems have an
    empty off-diagonal part (zero-size conversion, diagonal-only epilogue)."""
    kw = dict(matrix_f16=f16)
    A = gen.poisson7(5)
    S = ispm.PCGSolver(A, inner=inner, tol=1e-10, prec="fsai_gpu", **kw)
    x, st = S.solve_host(np.zeros(A.n_rows))
    assert st["converged"] and st["iterations"] == 0 and not np.any(x)
    one = ispm.csr_matrix(1, 1, np.array([0, 1], np.int32), np.array([0], np.int32),
                          np.array([4.0]))
    S1 = ispm.PCGSolver(one, inner=inner, tol=1e-10, prec="fsai_gpu", **kw)
    x1, st1 = S1.solve_host(np.array([2.0]))
    assert st1["converged"] and abs(x1[0] - 0.5) <= 1e-12
    # a diagonal system: its FSAI factor is D^(-1/2), exact when stored in
    # FP32 (one iteration); stored as FP16 x 2^k (the default) the
    # preconditioned matrix has eigenvalues within 2^-10 of 1, a few
    # iterations to 1e-10
    n = 1000
    d = np.arange(1, n + 1, dtype=np.float64)
    D = ispm.csr_matrix(n, n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), d)
    for fac16, most in ((False, 2), (None, 6)):
        SD = ispm.PCGSolver(D, inner=inner, tol=1e-10, prec="fsai_gpu", factor_f16=fac16, **kw)
        xd, std = SD.solve_host(d.copy())
        assert std["converged"] and std["iterations"] <= most, (fac16, std)
        assert np.allclose(xd, 1.0, rtol=0, atol=1e-9)
