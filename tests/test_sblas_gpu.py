"""sblas kernels on the GPU against the CPU oracle (util/cuda/sblas.cu).

Element-wise recurrences are bit-exact (both sides use the same fused
multiply-adds); reductions accumulate in FP64 on the GPU and in long double in
the oracle and must agree within 1e-13 of sum |terms| (FP64 vectors) or to the
rounding of the FP32 result (FP32 vectors)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = {np.float32: 0, np.float64: 1}


def tt(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("n", [0, 1, 3, 257, 4099, 1 << 20, (1 << 21) + 5])
@pytest.mark.parametrize("offset", [0, 1])
def test_dot(ispm, oracle, cuda, T, n, offset):
    rng = np.random.default_rng(n + offset)
    xa = rng.uniform(-1, 1, n + offset).astype(T)
    ya = rng.uniform(-1, 1, n + offset).astype(T)
    x, y = tt(cuda, xa)[offset:], tt(cuda, ya)[offset:]  # offset 1: unaligned vectors
    s = cuda.zeros(1, dtype=x.dtype, device="cuda")
    for same in (False, True):
        yy = x if same else y
        ispm.sblas.dot(x, yy, s, n)
        got = float(s.item())
        xs, ys = xa[offset:], (xa if same else ya)[offset:]
        exact = oracle.orc().orc_dot(DT[T], xs.ctypes.data, ys.ctypes.data, n)
        scale = float(np.abs(xs.astype(np.float64) * ys).sum())
        if T == np.float64:
            assert abs(got - exact) <= 1e-13 * max(scale, 1e-300)
        else:
            assert got == np.float32(exact) or abs(got - exact) <= 1e-6 * max(abs(exact), 1e-30)


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_dot_repeatable(ispm, cuda, T):
    x = cuda.rand(3_000_001, dtype=cuda.float64 if T == np.float64 else cuda.float32,
                  device="cuda")
    s = cuda.zeros(4, dtype=x.dtype, device="cuda")
    for k in range(4):
        ispm.sblas.dot(x, x, s[k:k + 1], x.numel())
    assert len(set(s.cpu().numpy().tolist())) == 1  # deterministic finish


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_update_scalars_bitexact(ispm, oracle, cuda, T):
    rng = np.random.default_rng(1)
    for _ in range(20):
        vals = rng.uniform(0.1, 10, 5).astype(T)
        al, be, ga, go, de = (tt(cuda, vals[i:i + 1].copy()) for i in range(5))
        ispm.sblas.ppcg_update_scalars(al, be, ga, go, de)
        o = vals.copy()
        oracle.orc().orc_ppcg_update_scalars(DT[T], o[0:].ctypes.data, o[1:].ctypes.data,
                                             o[2:].ctypes.data, o[3:].ctypes.data,
                                             o[4:].ctypes.data)
        assert al.item() == o[0] and be.item() == o[1]


@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("n", [1, 7, 1000, 65536 + 3, 1 << 22])
def test_update_vectors(ispm, oracle, cuda, T, n):
    rng = np.random.default_rng(n)
    host = {k: rng.standard_normal(n).astype(T) for k in "nmpsqzxruw"}
    alpha, beta = np.array([0.37], T), np.array([0.81], T)
    dev = {k: tt(cuda, v.copy()) for k, v in host.items()}
    red = cuda.zeros(3, dtype=dev["x"].dtype, device="cuda")
    ispm.sblas.ppcg_update_vectors(red[0:1], red[1:2], red[2:3], tt(cuda, alpha),
                                   tt(cuda, beta), dev["n"], dev["m"], dev["p"], dev["s"],
                                   dev["q"], dev["z"], dev["x"], dev["r"], dev["u"], dev["w"], n)
    o = {k: v.copy() for k, v in host.items()}
    ored = np.zeros(3)
    oracle.orc().orc_ppcg_update_vectors(DT[T], ored[0:].ctypes.data, ored[1:].ctypes.data,
                                         ored[2:].ctypes.data, alpha.ctypes.data,
                                         beta.ctypes.data, o["n"].ctypes.data,
                                         o["m"].ctypes.data,
                                         *[o[k].ctypes.data for k in "psqzxruw"], n)
    for k in "psqzxruw":
        assert np.array_equal(dev[k].cpu().numpy().view(np.uint8), o[k].view(np.uint8)), k
    r, u, w = (o[k].astype(np.float64) for k in "ruw")
    scales = (np.abs(r).sum(), np.abs(r * u).sum(), np.abs(w * u).sum())
    got = red.cpu().numpy().astype(np.float64)
    for g, e, sc in zip(got, ored, scales):
        tol = 1e-13 * sc if T == np.float64 else 1.2e-7 * max(abs(e), 1e-30) + 1e-13 * sc
        assert abs(g - e) <= tol


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_copy_and_add_indexed(ispm, oracle, cuda, T):
    rng = np.random.default_rng(9)
    n_src, n = 5000, 3000
    src = rng.standard_normal(n_src).astype(T)
    idx = rng.choice(n_src, n, replace=False).astype(np.int32)
    dst = cuda.zeros(n, dtype=cuda.float64 if T == np.float64 else cuda.float32, device="cuda")
    ispm.sblas.copy_indexed(dst, tt(cuda, src), tt(cuda, idx), n)
    assert np.array_equal(dst.cpu().numpy(), src[idx])
    # scatter-add with unique indices: exact
    base = rng.standard_normal(n_src).astype(T)
    d2 = tt(cuda, base.copy())
    vals = rng.standard_normal(n).astype(T)
    ispm.sblas.add_indexed(d2, tt(cuda, vals), tt(cuda, idx), n)
    o = base.copy()
    oracle.orc().orc_add_indexed(DT[T], o.ctypes.data, vals.ctypes.data, idx.ctypes.data, n)
    assert np.array_equal(d2.cpu().numpy(), o)
    # repeated indices all count (the reference races on them)
    rep = rng.integers(0, 17, n).astype(np.int32)
    d3 = cuda.zeros(17, dtype=d2.dtype, device="cuda")
    ispm.sblas.add_indexed(d3, tt(cuda, vals), tt(cuda, rep), n)
    o3 = np.zeros(17, T)
    oracle.orc().orc_add_indexed(DT[T], o3.ctypes.data, vals.ctypes.data, rep.ctypes.data, n)
    assert np.allclose(d3.cpu().numpy(), o3, rtol=1e-4 if T == np.float32 else 1e-12,
                       atol=1e-4 if T == np.float32 else 1e-12)
