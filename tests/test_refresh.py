"""Device-side value refresh for an unchanged sparsity pattern (the fast path
of plan/plan.h:39-56 update_device_matrix_coefs / change_host_matrix): the
CSR entry -> element slot map, and the scatter on the GPU."""
import numpy as np
import pytest

MODES = [(32, 1, 0, 1), (64, 1, 0, 0), (16, 2, 0, 0), (64, 4, 0, 0), (256, 1, 1, 0),
         (256, 1, 1, 1), (128, 2, 1, 0)]


@pytest.mark.parametrize("mode", MODES)
def test_value_map_places_every_entry(ispm, gen, mode):
    for A in (gen.poisson7(10), gen.stencil_grf(9, 27, 3.0, 1.5, 1),
              gen.random_csr(1500, 1500, 61, mean_len=9, pair_frac=0.6),
              gen.random_csr(700, 900, 62, mean_len=12, dtype=np.float32)):
        Ac = ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr.copy(), A.cols.copy(), A.elms.copy())
        B = ispm.csr_to_slell(Ac, *mode)
        m = ispm.slell_value_map(B, A)
        assert m.size == A.n_nz
        assert np.unique(m).size == m.size  # one slot per entry
        el = B.elms
        assert np.array_equal(el[m].view(np.uint8), A.elms.view(np.uint8))
        pad = np.ones(el.size, bool)
        pad[m] = False
        assert np.all(el[pad] == 0)  # every other slot is padding


def test_value_map_rejects_other_pattern(ispm, gen):
    A = gen.poisson7(8)
    B = ispm.csr_to_slell(ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr.copy(), A.cols.copy(),
                                          A.elms.copy()), 32, 1, False, True)
    other = gen.random_csr(A.n_rows, A.n_cols, 5, mean_len=7)
    with pytest.raises(ispm.IspmError):
        ispm.slell_value_map(B, other)


@pytest.mark.gpu
@pytest.mark.parametrize("E", [np.float64, np.float32])
def test_plan_refresh_values_on_device(ispm, oracle, cuda, gen, E):
    A = gen.stencil_grf(14, 27, 4.0, 1.5, 1)
    T = np.float64 if E == np.float64 else np.float32
    p = ispm.spmv_plan(A.astype(E), ispm.PLAN_DEFAULT, 0, T=T)
    # time step: same pattern, new coefficients (as FP64 device values)
    A2 = gen.stencil_grf(14, 27, 4.0, 1.5, 2)
    assert np.array_equal(A.row_ptr, A2.row_ptr) and np.array_equal(A.cols, A2.cols)
    vals = cuda.from_numpy(A2.elms.copy()).cuda()
    for _ in range(2):  # the second call reuses the cached map
        ispm.plan_refresh_values(p, A, vals)
    x = np.random.default_rng(3).uniform(-1, 1, A.n_cols).astype(T)
    n_pad = p.host_matrix.n_rows
    tdt = cuda.float64 if T == np.float64 else cuda.float32
    y = cuda.zeros(n_pad, dtype=tdt, device="cuda")
    p.execute_spmv(cuda.from_numpy(x).cuda(), y)
    A2e = A2.elms.astype(E).astype(np.float64)
    ref = oracle.csr_spmv_f64(A2.row_ptr, A2.cols, A2e, x.astype(np.float64))
    absr = oracle.csr_spmv_f64(A2.row_ptr, A2.cols, np.abs(A2e), np.abs(x.astype(np.float64)))
    err = np.linalg.norm(y.cpu().numpy()[: A.n_rows].astype(np.float64) - ref)
    assert err <= (1e-14 if E == np.float64 else 1e-6) * np.linalg.norm(absr)
