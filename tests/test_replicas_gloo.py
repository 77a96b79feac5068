"""Multi-rank host logic on CPU (gloo, world size 2 and 3): the balanced
sharding of the Monte-Carlo realisations, max / sum over ranks and the
all-gather of per-rank results, with each rank stepping its share of a small
noise-free SH chain on the CPU oracle and the gathered slopes checked
against a single-process run."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from specula_b200.replicas import partition, shard_groups


def test_partition_is_balanced_and_complete():
    for n in (0, 1, 5, 96, 97):
        for ws in (1, 2, 3, 8):
            parts = [list(partition(n, ws, r)) for r in range(ws)]
            assert sum(parts, []) == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        partition(4, 2, 2)


def test_shard_groups_keeps_every_realisation_once():
    groups = [('a', list(range(55))), ('b', list(range(100, 127))), ('c', list(range(200, 214)))]
    for ws in (1, 2, 3, 8, 20):
        seen = []
        for r in range(ws):
            mine = shard_groups(groups, ws, r)
            for tmpl, reals in mine:
                assert reals
                seen += [(tmpl, x) for x in reals]
        assert sorted(seen) == sorted((t, x) for t, rs in groups for x in rs)


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _slopes_of(seed):
    """Noise-free SH + CoG on the CPU oracle for one seeded phase."""
    from oracle import sh as osh, slopec as osl
    from oracle.masks import make_mask
    g = osh.sh_geometry(750.0, 6 * 0.3867, 0.3867, 8, 6, 64, 0.05, fov_ovs_coeff=1.0)
    A = make_mask(64, 0.14, 1.0).astype(np.float32)
    ph = (np.random.default_rng(seed).standard_normal((64, 64)) * 40).astype(np.float32) * A
    frame = osh.SHOracle(g, 750.0, precision=1).forward(A, ph, 5.0, 0.05)
    flat = osh.SHOracle(g, 750.0, precision=1).forward(A, np.zeros_like(ph), 5.0, 0.05)
    idxs, _ = osl.detect_subaps(flat, 8, 0.5)
    return osl.sh_slopes(frame, idxs, precision=1)[0]


def _rank_main(rank, ws, port, seeds, q):
    import torch.distributed as dist
    from specula_b200 import replicas
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    import datetime
    dist.init_process_group('gloo', rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        r, w = replicas.world()
        assert (r, w) == (rank, ws)
        mine = [seeds[i] for i in replicas.partition(len(seeds), ws, rank)]
        local = {s: _slopes_of(s) for s in mine}
        tmax = replicas.max_over_ranks(10.0 + rank)
        tsum = replicas.sum_over_ranks(float(len(mine)))
        gathered = replicas.gather_objects(local)
        dist.barrier()
        if rank == 0:
            merged = {}
            for d in gathered:
                assert not set(d) & set(merged)
                merged.update(d)
            q.put((tmax, tsum, {k: v.tolist() for k, v in merged.items()}))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('ws', [2, 3])
def test_ranks_shard_step_and_gather(ws):
    seeds = [11, 12, 13, 14, 15]
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, seeds, q)) for r in range(ws)]
    for p in procs:
        p.start()
    try:
        tmax, tsum, merged = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
    for p in procs:
        assert p.exitcode == 0
    assert tmax == 10.0 + ws - 1
    assert tsum == len(seeds)
    assert sorted(merged) == seeds
    for s in seeds:
        assert np.array_equal(np.array(merged[s], dtype=np.float32), _slopes_of(s))
