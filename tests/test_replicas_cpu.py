"""World-size-2 test of the replica path on CPU (gloo): each rank runs its own
transform (CPU oracle here, the rank logic is what is under test), the job
time is the max over ranks and the pair count the sum."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from oracle import oracle as O
    from s2dw_b200 import replicas
    from s2dw_b200.workload import gaussian_flm

    w, r, _ = replicas.init_group("gloo", timeout_s=60)
    assert (w, r) == (world, rank)
    B, N, alpha = 16, 2, 2.0
    J = O.comp_jmax(B, alpha)
    K, P, bs = O.init_kernels(J, B, alpha)
    S = O.init_directionality(B, N)
    flm = gaussian_flm(B, seed=100 + rank)  # each replica its own map
    wav, sc = O.analysis_dynamic(flm, K, S, J, B, N, bs, alpha)
    f2 = O.synthesis_dynamic(wav, sc, K, P, S, J, B, N, bs, alpha)
    err = float(np.abs(f2 - flm).max())
    replicas.barrier(w)
    elapsed = 1.0 + rank  # stand-in per-rank time
    tmax = replicas.max_over_ranks(elapsed, w)
    pairs = replicas.sum_over_ranks(1, w)
    emax = replicas.max_over_ranks(err, w)
    out[rank] = (tmax, pairs, emax)
    replicas.finish(w)


def test_two_rank_replicas_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    assert res[0] == res[1]
    tmax, pairs, emax = res[0]
    assert tmax == 2.0 and pairs == 2.0 and emax < 1e-12
