"""Multi-rank batched solves: systems are sharded across ranks by LPT with
no data-path collective; the ranks' per-system results are gathered on the
host.  Run here as two gloo ranks on CPU, each solving its shard with the
FP64 CPU oracle (the GPU batched solver takes the same place on a GPU
rank)."""
import os
import socket

import numpy as np
import pytest


def test_lpt_partition_properties(ispm):
    rng = np.random.default_rng(0)
    costs = list(rng.lognormal(0, 1, 97))
    for world in (1, 2, 3, 8):
        shards = ispm.shard_lpt(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shards]
        # LPT bound: makespan <= 4/3 of the optimum, which is at least
        # max(mean load, largest job)
        assert max(loads) <= 4 / 3 * max(sum(costs) / world, max(costs)) + 1e-9
    # deterministic, ties to the lowest rank
    assert ispm.shard_lpt([1, 1, 1, 1], 2) == [[0, 2], [1, 3]]


def _solve_cpu(systems, bs, oracle, idx):
    out = {}
    for k in idx:
        A = systems[k]
        g = oracle.fsai_lower_f64(A.row_ptr, A.cols, A.elms)
        import scipy.sparse as sp
        Gs = sp.csr_matrix((g[2], g[1], g[0]), shape=(A.n_rows, A.n_rows))
        Gt = Gs.T.tocsr()
        its = []
        for b in bs[k]:
            x, it, rel = oracle.pcg_f64((A.row_ptr, A.cols, A.elms), b,
                                        (g[0], g[1], g[2]),
                                        (Gt.indptr.astype(np.int32), Gt.indices.astype(np.int32),
                                         Gt.data), tol=1e-8)
            assert rel <= 1e-8 * 1.001
            its.append(int(it))
        out[k] = its
    return out


def _rank_main(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (os.path.join(root, "ispm-sparse-lib_b200"), os.path.join(root, "oracle")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    import ispm.gen as gen
    import ispm.shard as shard
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        systems, n_rhs, _ = gen.batch_systems(6, seed=2, lo=4, hi=7)
        _, bs = gen.batch_rhs(systems, n_rhs, seed=3)
        mine, merged = shard.run_sharded(
            systems, n_rhs, lambda idx: _solve_cpu(systems, bs, oracle, idx), rank, world,
            gather=dist.all_gather_object)
        q.put((rank, mine, merged))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_batch_two_gloo_ranks(ispm, gen, oracle):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    systems, n_rhs, _ = gen.batch_systems(6, seed=2, lo=4, hi=7)
    _, bs = gen.batch_rhs(systems, n_rhs, seed=3)
    serial = _solve_cpu(systems, bs, oracle, range(len(systems)))
    mine0, mine1 = got[0][1], got[1][1]
    assert sorted(mine0 + mine1) == list(range(len(systems)))
    assert not set(mine0) & set(mine1)
    # every rank holds the full gathered result, equal to the serial one
    assert got[0][2] == got[1][2] == serial
