"""Tile records of the staged SpMV walk (ispm_slell_stage_records), checked
on the host against a numpy restatement of the kernel's indexing
(csrc/spmv_staged.cuh): for every staged tile, every slice's k-th diagonal
is the k-th set bit of its mask, and every thread's four x values (tile rows
4 tid .. 4 tid + 3) come from the two shared-memory chunks the kernel reads,
which hold x[w + t] (zero outside x) and lie inside the copied bands;
windows are grouped by their shift modulo 4."""
import numpy as np
import pytest

TILE = 1024


def check_records(B):
    v = B.view()
    S, sp = v.slice_height, B.slice_ptr.astype(np.int64)
    recs = B.stage_records()
    spt = TILE // S
    assert recs.shape == ((v.n_slices + spt - 1) // spt, 224)
    staged = 0
    for tile, r in enumerate(recs):
        if not r[0]:
            continue
        staged += 1
        b0 = tile * spt
        nsl = min(spt, v.n_slices - b0)
        nb, total, nu = r[1], r[2], r[3]
        assert 1 <= nb <= 8 and total % 4 == 0 and 1 <= nu <= 64
        # shared-memory word -> absolute x column, band by band as copied
        col_of = np.full(total, np.iinfo(np.int64).min)
        prev = 0
        for q in range(nb):
            c0, run, dst0 = r[4 + 3 * q], r[5 + 3 * q], r[6 + 3 * q]
            nch = run - prev
            prev = run
            assert c0 % 4 == 0 and nch >= 1
            assert dst0 >= 0 and dst0 % 4 == 0 and dst0 + nch * 4 <= total
            assert np.all(col_of[dst0: dst0 + nch * 4] == np.iinfo(np.int64).min)  # no overlap
            col_of[dst0: dst0 + nch * 4] = c0 + np.arange(nch * 4)
        ends = [r[28 + m] for m in range(4)]
        assert ends == sorted(ends) and ends[3] == nu
        sx_of = {}
        for m in range(4):
            for i in range(ends[m - 1] if m else 0, ends[m]):
                e = int(r[32 + i])
                sx, u = e & 0xFFFFFF, e >> 24
                assert sx % 4 == m and u not in sx_of
                sx_of[u] = sx
        assert sorted(sx_of) == list(range(nu))
        for s in range(nsl):
            b = b0 + s
            nd = (sp[3 * b + 3] - sp[3 * b] - (sp[3 * b + 4] - sp[3 * b + 1])) // S
            mask = (int(r[97 + 2 * s]) & 0xFFFFFFFF) << 32 | (int(r[96 + 2 * s]) & 0xFFFFFFFF)
            bits = [u for u in range(64) if mask >> u & 1]
            assert len(bits) == nd
            if r[0] == 1:  # uniform tile: the kernel takes window u as diagonal k = u
                assert bits == list(range(nu))
            else:
                assert r[0] == 2
            tid = (s * S + np.arange(0, S, 4)) // 4  # threads of the slice
            for k, u in enumerate(bits):
                dp = int(sp[sp[3 * b + 2] + k])  # diag_pos: local row r reads x[dp + r - S]
                sx = sx_of[u]
                q = (sx >> 2) + tid
                assert q.min() >= 0 and 4 * (q.max() + 2) <= total + 4
                words = np.concatenate([4 * q[:, None] + np.arange(8)], axis=0)
                shift = sx % 4
                need = words[:, shift: shift + 4]
                t = 4 * tid[:, None] + np.arange(4)  # tile rows
                local = t - s * S                     # rows within the slice
                assert np.array_equal(col_of[need], dp + local - S), (tile, s, k)
                if shift:  # the second chunk the kernel loads lies inside a band
                    assert np.all(col_of[4 * (q + 1)] != np.iinfo(np.int64).min)
    return staged, len(recs)


@pytest.mark.parametrize("S", [16, 32, 64, 128, 256, 512])
def test_stage_records_stencils(ispm, gen, S):
    for A in (gen.poisson7(24), gen.stencil_grf(20, 27, 4.0, 1.5, 2), gen.poisson7(32)):
        staged, n = check_records(ispm.csr_to_slell(A, S, 1, 0, 1))
        # with slice masks every tile of a stencil matrix stages
        assert staged == n, (staged, n)


def test_stage_records_irregular(ispm, gen):
    import scipy.sparse as sp
    # a banded random matrix: slices carry different diagonal sets
    n = 5000
    rng = np.random.default_rng(3)
    offs = [-40, -7, -1, 0, 1, 7, 40]
    M = sp.diags([rng.uniform(-1, 1, n - abs(o)) for o in offs], offs, format="csr")
    keep = rng.uniform(size=M.nnz) < 0.8
    M.data[~keep] = 0.0
    M.eliminate_zeros()
    M.sort_indices()
    A = ispm.csr_matrix(n, n, M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data)
    for S in (32, 64):
        check_records(ispm.csr_to_slell(A, S, 1, 0, 1))


def test_stage_records_only_for_the_staged_formats(ispm, gen):
    A = gen.poisson7(10)
    assert ispm.csr_to_slell(A, 64, 1, 0, 0).stage_records().size == 0  # no diagonals
    assert ispm.csr_to_slell(A, 64, 2, 0, 0).stage_records().size == 0  # hblocks
    assert ispm.csr_to_slell(A, 64, 1, 1, 1).stage_records().size == 0  # variable height
