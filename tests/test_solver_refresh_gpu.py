"""ispm_solver_update_values: a solver created with opts.refresh on A1 takes
the values of A2 (same pattern) on the device and must then solve exactly as
a solver created on A2 does -- same iteration count, same solution to
rounding of the FP64 solution (the device factor is rebuilt from the same
values by the same kernels) -- with natural and renumbered (RCM) orders,
FP32 and FP64 inner iterations, FP16 factors, host and device values, and a
given factor pair (which stays as given).  Every solve is also judged by its
true residual against the FP64 CSR oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def with_values(ispm, A, vals):
    return ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr, A.cols,
                           np.ascontiguousarray(vals, np.float64))


def solve(oracle, S, A, b, tol):
    x, st = S.solve_host(b)
    assert st["converged"], st
    r = b - oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= tol * 1.001
    return x, st


def pair(gen, ispm, k):
    """Two systems with one pattern: GRF couplings from two seeds."""
    A1 = gen.stencil_grf(k, 27, 4.0, 1.5, 1)
    A2 = gen.stencil_grf(k, 27, 4.0, 1.5, 2)
    assert np.array_equal(A1.row_ptr, A2.row_ptr) and np.array_equal(A1.cols, A2.cols)
    return A1, A2


@pytest.mark.parametrize("inner,f16", [(np.float32, False), (np.float64, False),
                                       (np.float32, True)], ids=["mixed", "fp64", "f16factor"])
@pytest.mark.parametrize("device_values", [False, True], ids=["host", "device"])
def test_update_matches_a_fresh_solver(ispm, oracle, cuda, gen, inner, f16, device_values):
    torch = cuda
    A1, A2 = pair(gen, ispm, 24)
    b = np.random.default_rng(3).uniform(-1, 1, A1.n_rows)
    kw = dict(inner=inner, tol=1e-10, prec="fsai_gpu", factor_f16=f16)
    S = ispm.PCGSolver(A1, refresh=True, **kw)
    solve(oracle, S, A1, b, 1e-10)
    vals = torch.from_numpy(A2.elms.copy()).cuda() if device_values else A2.elms
    S.update_values(vals)
    x_up, st_up = solve(oracle, S, A2, b, 1e-10)
    x_new, st_new = solve(oracle, ispm.PCGSolver(A2, **kw), A2, b, 1e-10)
    assert st_up["iterations"] == st_new["iterations"], (st_up, st_new)
    assert np.allclose(x_up, x_new, rtol=0, atol=1e-13 * np.abs(x_new).max())
    # and back: the first system's solve again
    S.update_values(A1.elms)
    solve(oracle, S, A1, b, 1e-10)


@pytest.mark.parametrize("inner", [np.float32, np.float64])
def test_update_of_a_renumbered_solve(ispm, oracle, cuda, gen, inner):
    """A randomly numbered mesh, renumbered inside the solver (RCM): the new
    values arrive in the caller's order and are permuted on the device."""
    A1 = gen.unstructured(16, 0.05, 3, 0.1, 10.0, 1.01)
    rng = np.random.default_rng(8)
    # new symmetric values on the same pattern: scale every entry a_ij by
    # w_i w_j (w > 0), which keeps A SPD
    w = rng.uniform(0.5, 2.0, A1.n_rows)
    rows = np.repeat(np.arange(A1.n_rows), np.diff(A1.row_ptr))
    A2 = with_values(ispm, A1, A1.elms * w[rows] * w[A1.cols])
    b = rng.uniform(-1, 1, A1.n_rows)
    kw = dict(inner=inner, tol=1e-10, prec="fsai_gpu", reorder="rcm")
    S = ispm.PCGSolver(A1, refresh=True, **kw)
    solve(oracle, S, A1, b, 1e-10)
    S.update_values(A2.elms)
    x_up, st_up = solve(oracle, S, A2, b, 1e-10)
    x_new, st_new = solve(oracle, ispm.PCGSolver(A2, **kw), A2, b, 1e-10)
    assert st_up["iterations"] == st_new["iterations"], (st_up, st_new)
    assert np.allclose(x_up, x_new, rtol=0, atol=1e-13 * np.abs(x_new).max())


def test_update_keeps_a_given_pair(ispm, oracle, cuda, gen):
    """prec = given: only A changes; the solve equals a fresh solver on A2
    with the pair built for A1."""
    A1, A2 = pair(gen, ispm, 16)
    G1, G2 = ispm.fastainv_sym(A1, np.float64, None, 8_000_000, 0.01)
    b = np.random.default_rng(4).uniform(-1, 1, A1.n_rows)
    S = ispm.PCGSolver(A1, G1, G2, inner=np.float32, tol=1e-10, refresh=True)
    S.update_values(A2.elms)
    x_up, st_up = solve(oracle, S, A2, b, 1e-10)
    x_new, st_new = solve(oracle, ispm.PCGSolver(A2, G1, G2, inner=np.float32, tol=1e-10),
                          A2, b, 1e-10)
    assert st_up["iterations"] == st_new["iterations"]
    assert np.allclose(x_up, x_new, rtol=0, atol=1e-13 * np.abs(x_new).max())


def test_update_needs_refresh_and_no_f16_split(ispm, cuda, gen):
    A = gen.poisson7(8)
    S = ispm.PCGSolver(A, inner=np.float32, prec="fsai_gpu")
    with pytest.raises(ispm.IspmError):
        S.update_values(A.elms)
    with pytest.raises(ispm.IspmError):
        ispm.PCGSolver(A, inner=np.float32, prec="fsai_gpu", matrix_f16=True, refresh=True)
