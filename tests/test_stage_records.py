"""Tile records of the staged SpMV walk (ispm_slell_stage_records), checked
on the host against a numpy restatement of the kernel's indexing
(csrc/spmv_staged.cuh): for every staged tile, the copy list names the
tile's element range and x bands (16-byte aligned), every slice's k-th
diagonal is the k-th set bit of its mask, its elements sit where the
compute warps read them (uniform tiles: slice s, window u at s nu S + u S),
its explicit-column entries sit just before them, and tile row t of a slice
reads x-area word [8 + u] + t, which holds the x column diag_pos + r - S the
reference walk reads for local row r."""
import numpy as np
import pytest

TILE = 256
EMPTY = np.iinfo(np.int64).min


def check_records(B):
    v = B.view()
    S, sp = v.slice_height, B.slice_ptr.astype(np.int64)
    recs = B.stage_records()
    spt = TILE // S
    assert recs.shape == ((v.n_slices + spt - 1) // spt, 176)
    staged = 0
    for tile, r in enumerate(recs):
        b0 = tile * spt
        nsl = min(spt, v.n_slices - b0)
        assert r[2] == nsl
        if not r[0]:
            continue
        assert r[0] in (1, 2)
        staged += 1
        nu, nb, words = r[1], r[154], r[155]
        assert 1 <= nu <= 64 and 1 <= nb <= 8 and words % 4 == 0 and words <= 8192
        # the copy list: elements of the whole tile, then the bands
        assert r[152] == sp[3 * b0] and r[153] == sp[3 * (b0 + nsl)] - sp[3 * b0]
        col_of = np.full(words, EMPTY)
        dst = 0
        for q in range(nb):
            c0, w = r[156 + 2 * q], r[157 + 2 * q]
            assert c0 % 4 == 0 and w % 4 == 0 and w > 0
            col_of[dst: dst + w] = c0 + np.arange(w)
            dst += w
        assert dst == words
        for s in range(nsl):
            b = b0 + s
            e0, c0, dd, e1, c1 = (int(z) for z in sp[3 * b: 3 * b + 5])
            ne = (c1 - c0) // S
            nd = (e1 - e0) // S - ne
            mask = (int(r[73 + 2 * s]) & 0xFFFFFFFF) << 32 | (int(r[72 + 2 * s]) & 0xFFFFFFFF)
            bits = [u for u in range(64) if mask >> u & 1]
            assert len(bits) == nd and max(bits, default=-1) < nu
            # explicit-column entries: count, columns, elements before the diagonals
            assert r[120 + s] == ne and r[136 + s] == c0
            assert r[104 + s] == e0 + ne * S - r[152]
            if r[0] == 1:
                assert ne == 0 and bits == list(range(nu)) and r[104 + s] == s * nu * S
            t = s * S + np.arange(S)          # tile rows of the slice
            for k, u in enumerate(bits):
                dp = int(sp[dd + k])          # diag_pos: local row r reads x[dp + r - S]
                words_read = r[8 + u] + t
                assert words_read.min() >= 0 and words_read.max() < words
                assert np.array_equal(col_of[words_read], dp + np.arange(S) - S), (tile, s, k)
                # the element the compute warp reads for (row, diagonal k)
                off = (s * nu * S + u * S) if r[0] == 1 else (r[104 + s] + k * S)
                assert off + r[152] == e0 + ne * S + k * S
    return staged, len(recs)


@pytest.mark.parametrize("S", [16, 32, 64, 128, 256])
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
        staged, n_tiles = check_records(ispm.csr_to_slell(A, S, 1, 0, 1))
        assert staged > 0


def test_stage_records_only_for_the_staged_formats(ispm, gen):
    A = gen.poisson7(10)
    assert ispm.csr_to_slell(A, 64, 1, 0, 0).stage_records().size == 0  # no diagonals
    assert ispm.csr_to_slell(A, 64, 2, 0, 0).stage_records().size == 0  # hblocks
    assert ispm.csr_to_slell(A, 64, 1, 1, 1).stage_records().size == 0  # variable height
    assert ispm.csr_to_slell(A, 512, 1, 0, 1).stage_records().size == 0  # taller than a tile
