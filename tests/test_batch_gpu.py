"""Batched PCG (ispm_batch_*): many independent SPD systems of uneven size,
1-4 right-hand sides each, advanced by one set of launches per iteration.

The reference has no batched solver; a caller runs its primitives
(cuda/spmv/kernel-iface.h:20-74, util/cuda/sblas.cu:156-237) once per
system.  Every lane's solution is judged against the FP64 CSR oracle by its
true residual, and against the single-system solver (same method, one
system at a time) by iteration count."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _true_rel(oracle, A, x, b):
    r = b - oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, x)
    return np.linalg.norm(r) / np.linalg.norm(b)


def _small_batch(gen, n=7, seed=3, lo=6, hi=20):
    return gen.batch_systems(n, seed=seed, lo=lo, hi=hi)


@pytest.mark.parametrize("inner", [np.float32, np.float64])
def test_batch_residuals(ispm, oracle, cuda, gen, inner):
    systems, n_rhs, dims = _small_batch(gen)
    _, bs = gen.batch_rhs(systems, n_rhs, seed=1)
    B = ispm.BatchSolver(systems, n_rhs, inner=inner, tol=1e-8)
    assert B.lanes == sum(n_rhs)
    xs, lanes, tot = B.solve_host(bs)
    assert tot["converged"], lanes
    for lane in range(B.lanes):
        info = B.lane_info(lane)
        k, j = info["system"], info["rhs"]
        rel = _true_rel(oracle, systems[k], xs[k][j], bs[k][j])
        assert lanes[lane]["converged"] and lanes[lane]["true_relres"] <= 1e-8
        # the reported residual is the FP64 one the oracle computes
        assert rel <= 1e-8 * 1.001
        assert abs(rel - lanes[lane]["true_relres"]) <= 1e-3 * 1e-8 + 1e-3 * rel
    assert B.launches > 0


def test_batch_matches_single_solver(ispm, oracle, cuda, gen):
    """Same method lane by lane: iteration counts of the batched lanes agree
    with the single-system classic PCG + GPU FSAI solve of that system."""
    systems, n_rhs, _ = _small_batch(gen, n=5, seed=7)
    _, bs = gen.batch_rhs(systems, n_rhs, seed=2)
    B = ispm.BatchSolver(systems, n_rhs, inner=np.float64, tol=1e-8)
    xs, lanes, tot = B.solve_host(bs)
    assert tot["converged"]
    for lane in range(B.lanes):
        info = B.lane_info(lane)
        k, j = info["system"], info["rhs"]
        S = ispm.PCGSolver(systems[k], inner=np.float64, tol=1e-8, prec="fsai_gpu",
                           variant="classic")
        x1, st = S.solve_host(bs[k][j])
        assert st["converged"]
        # iteration counts within the reliable-update granularity
        assert abs(lanes[lane]["iterations"] - st["iterations"]) <= 0.1 * st["iterations"] + 4
        assert np.allclose(xs[k][j], x1, rtol=0, atol=1e-6 * np.abs(x1).max())


def test_batch_groups_and_lane_layout(ispm, cuda, gen):
    systems, n_rhs, dims = _small_batch(gen, n=9, seed=11)
    B = ispm.BatchSolver(systems, n_rhs, inner=np.float32)
    groups = B.groups()
    assert sum(l for _, l in groups) == B.lanes
    seen = set()
    prev_end = 0
    for lane in range(B.lanes):
        info = B.lane_info(lane)
        assert info["row0"] % 1024 == 0 and info["row0"] >= prev_end
        n = systems[info["system"]].n_rows
        prev_end = info["row0"] + -(-n // 1024) * 1024
        seen.add((info["system"], info["rhs"]))
    assert prev_end == B.rows
    assert seen == {(k, j) for k in range(len(systems)) for j in range(n_rhs[k])}


def test_batch_uneven_stop_and_zero_rhs(ispm, oracle, cuda, gen):
    """A zero right-hand side finishes at once with x = 0; an easy lane (tiny
    system) stops long before a hard one and both meet the tolerance."""
    easy = gen.poisson7(4)                      # 64 rows
    hard = gen.lognormal_stencil(24, 27, 1.5, 5)  # 13,824 rows
    rng = np.random.default_rng(0)
    b_easy = rng.uniform(-1, 1, (2, easy.n_rows))
    b_easy[1] = 0.0
    b_hard = rng.uniform(-1, 1, (1, hard.n_rows))
    B = ispm.BatchSolver([easy, hard], [2, 1], inner=np.float32, tol=1e-9)
    xs, lanes, tot = B.solve_host([b_easy, b_hard])
    assert tot["converged"], lanes
    by = {(B.lane_info(l)["system"], B.lane_info(l)["rhs"]): lanes[l] for l in range(3)}
    assert by[(0, 1)]["iterations"] == 0 and not np.any(xs[0][1])
    assert by[(0, 0)]["iterations"] < by[(1, 0)]["iterations"]
    assert _true_rel(oracle, easy, xs[0][0], b_easy[0]) <= 1e-9 * 1.001
    assert _true_rel(oracle, hard, xs[1][0], b_hard[0]) <= 1e-9 * 1.001


def test_batch_no_prec_and_graph_off(ispm, oracle, cuda, gen):
    """Without a preconditioner, and with the iteration chunks launched one
    kernel at a time instead of as a graph: the same results bit for bit
    (all lane sums are formed in a fixed order)."""
    systems, n_rhs, _ = _small_batch(gen, n=4, seed=5, lo=6, hi=14)
    _, bs = gen.batch_rhs(systems, n_rhs, seed=4)
    out = []
    for use_graph in (True, False):
        B = ispm.BatchSolver(systems, n_rhs, inner=np.float32, tol=1e-8, prec="none",
                             use_graph=use_graph)
        xs, lanes, tot = B.solve_host(bs)
        assert tot["converged"]
        out.append((xs, [l["iterations"] for l in lanes]))
    assert out[0][1] == out[1][1]
    for a, b in zip(out[0][0], out[1][0]):
        assert np.array_equal(a, b)


def test_batch_device_vectors(ispm, oracle, cuda, gen):
    """ispm_batch_solve on stacked device vectors (lane l at row0)."""
    import torch
    systems, n_rhs, _ = _small_batch(gen, n=3, seed=9)
    _, bs = gen.batch_rhs(systems, n_rhs, seed=6)
    B = ispm.BatchSolver(systems, n_rhs, inner=np.float32, tol=1e-8)
    bh = np.zeros(B.rows)
    for lane in range(B.lanes):
        info = B.lane_info(lane)
        b = bs[info["system"]][info["rhs"]]
        bh[info["row0"]:info["row0"] + b.size] = b
    bd = torch.tensor(bh, device="cuda")
    xd = torch.empty_like(bd)
    lanes, tot = B.solve(bd, xd)
    torch.cuda.synchronize()
    xh = xd.cpu().numpy()
    assert tot["converged"]
    for lane in range(B.lanes):
        info = B.lane_info(lane)
        k, j = info["system"], info["rhs"]
        n = systems[k].n_rows
        x = xh[info["row0"]:info["row0"] + n]
        assert _true_rel(oracle, systems[k], x, bs[k][j]) <= 1e-8 * 1.001
        # padding rows stay zero
        pad = xh[info["row0"] + n:info["row0"] + -(-n // 1024) * 1024]
        assert not np.any(pad)


def test_batch_rejects_bad_args(ispm, cuda, gen):
    A = gen.poisson7(4)
    with pytest.raises(ispm.IspmError):
        ispm.BatchSolver([A], [0])
    with pytest.raises(ispm.IspmError):
        ispm.BatchSolver([A], [1], check_every=0)


def test_batch_single_lane_and_tiny_system(ispm, oracle, cuda, gen):
    """One lane only, and a 1 x 1 system next to a larger one."""
    A = gen.lognormal_stencil(10, 7, 1.0, 8)
    b = np.random.default_rng(1).uniform(-1, 1, A.n_rows)
    B = ispm.BatchSolver([A], 1, inner=np.float32, tol=1e-9)
    xs, lanes, tot = B.solve_host([b])
    assert tot["converged"] and B.lanes == 1
    r = b - oracle.csr_spmv_f64(A.row_ptr, A.cols, A.elms, xs[0])
    assert np.linalg.norm(r) <= 1e-9 * 1.001 * np.linalg.norm(b)
    one = ispm.csr_matrix(1, 1, np.array([0, 1], np.int32), np.array([0], np.int32),
                          np.array([4.0]))
    B2 = ispm.BatchSolver([one, A], [1, 1], inner=np.float64, tol=1e-9)
    xs2, lanes2, tot2 = B2.solve_host([np.array([2.0]), b])
    assert tot2["converged"], lanes2
    assert abs(xs2[0][0] - 0.5) <= 1e-12


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_batch_non_finite_rhs_stops_only_its_lane(ispm, oracle, cuda, gen, bad):
    """A lane whose right-hand side holds NaN / Inf stops at once with
    ERR_INVALID in its own status; every other lane still converges."""
    systems, n_rhs, dims = _small_batch(gen, n=4, seed=5)
    _, bs = gen.batch_rhs(systems, n_rhs, seed=2)
    bs = [b.copy() for b in bs]
    bs[1].reshape(-1)[3] = bad
    B = ispm.BatchSolver(systems, n_rhs, inner=np.float32, tol=1e-8)
    xs, lanes, tot = B.solve_host(bs)
    assert not tot["converged"]
    for lane in range(B.lanes):
        info = B.lane_info(lane)
        k, j = info["system"], info["rhs"]
        b = bs[k].reshape(n_rhs[k], -1)[j]
        if not np.all(np.isfinite(b)):
            assert lanes[lane]["status"] == ispm.ERR_INVALID and not lanes[lane]["converged"]
            assert lanes[lane]["iterations"] == 0
        else:
            assert lanes[lane]["converged"], (lane, lanes[lane])
            x = xs[k].reshape(n_rhs[k], -1)[j]
            assert _true_rel(oracle, systems[k], x, b) <= 1e-8 * 1.001
