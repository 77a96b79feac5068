"""One system split by bands of lenslet rows (specula_b200.rowband), host
logic on CPU: the bands and the mirror's column ranges, and, on gloo ranks
(world size 2 and 3), the exchange the split relies on: every rank keeps the
slope / flux entries of its own sub-apertures and the mirror phase of its own
rows, zero elsewhere, and the sum over the ranks is the one-process result
bit for bit (CPU oracle chain, noise-free)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from specula_b200.rowband import lenslet_bands, mirror_columns

N_LENSES, NPX, PIX = 8, 6, 64


def test_lenslet_bands_are_contiguous_balanced_and_complete():
    for n in (8, 20, 80):
        for ws in (1, 2, 3, 8):
            b = lenslet_bands(n, ws)
            rows = sum([list(range(r0, r0 + k)) for r0, k in b], [])
            assert rows == list(range(n))
            assert max(k for _, k in b) - min(k for _, k in b) <= 1
    with pytest.raises(ValueError):
        lenslet_bands(4, 5)


def test_mirror_columns_cover_every_mask_pixel_once():
    from oracle.masks import make_mask
    side = 64
    idx = np.flatnonzero(make_mask(side, 0.14, 1.0))
    for ws in (1, 2, 3, 8):
        owned = np.zeros(idx.size, dtype=int)
        for r0, k in lenslet_bands(N_LENSES, ws):
            c0, c1 = mirror_columns(idx, side, r0 * 8, (r0 + k) * 8)
            assert c0 % 4 == 0
            rows = idx[c0:c1] // side
            # the range starts at most 3 columns early (the previous band's pixels)
            assert np.all(rows[3:] >= r0 * 8) and np.all(rows < (r0 + k) * 8)
            owned[c0:c1][rows >= r0 * 8] += 1
        assert np.all(owned == 1)


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _system(seed):
    """Noise-free SH + CoG (CPU oracle) of a seeded phase, the sub-aperture
    table and a seeded mirror: (slopes, flux, lenslet row per sub-aperture,
    mirror mask indices, influence functions, commands)."""
    from oracle import sh as osh, slopec as osl
    from oracle.masks import make_mask
    g = osh.sh_geometry(750.0, 6 * 0.3867, 0.3867, N_LENSES, NPX, PIX, 0.05, fov_ovs_coeff=1.0)
    A = make_mask(PIX, 0.14, 1.0).astype(np.float32)
    rng = np.random.default_rng(seed)
    ph = (rng.standard_normal((PIX, PIX)) * 40).astype(np.float32) * A
    frame = osh.SHOracle(g, 750.0, precision=1).forward(A, ph, 5.0, 0.05)
    flat = osh.SHOracle(g, 750.0, precision=1).forward(A, np.zeros_like(ph), 5.0, 0.05)
    idxs, _ = osl.detect_subaps(flat, N_LENSES, 0.5)
    slopes, flux = osl.sh_slopes(frame, idxs, precision=1)
    lens_row = (idxs[:, 0] // (N_LENSES * NPX)) // NPX
    mask_idx = np.flatnonzero(A)
    IF = rng.standard_normal((12, mask_idx.size)).astype(np.float32)
    cmd = rng.standard_normal(12).astype(np.float32)
    return slopes, flux, lens_row, mask_idx, IF, cmd


def _phase(mask_idx, IF, cmd, c0, c1):
    out = np.zeros(PIX * PIX, dtype=np.float32)
    out[mask_idx[c0:c1]] = cmd @ IF[:, c0:c1]
    return out


def _rank_main(rank, ws, port, seed, q):
    import datetime
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        slopes, flux, lens_row, mask_idx, IF, cmd = _system(seed)
        r0, k = lenslet_bands(N_LENSES, ws)[rank]
        mine = (lens_row >= r0) & (lens_row < r0 + k)
        nv = flux.size
        # exchange 2: this rank's sub-apertures' slopes and flux, zero elsewhere
        vec = np.zeros(3 * nv, dtype=np.float32)
        vec[:nv][mine] = slopes[:nv][mine]
        vec[nv:2 * nv][mine] = slopes[nv:][mine]
        vec[2 * nv:][mine] = flux[mine]
        t = torch.as_tensor(vec)
        dist.all_reduce(t)
        # the mirror: this rank's columns, kept on its own rows
        c0, c1 = mirror_columns(mask_idx, PIX, r0 * 8, (r0 + k) * 8)
        ph = _phase(mask_idx, IF, cmd, c0, c1).reshape(PIX, PIX)
        own = np.zeros_like(ph)
        own[r0 * 8:(r0 + k) * 8] = ph[r0 * 8:(r0 + k) * 8]
        tp = torch.as_tensor(own)
        dist.all_reduce(tp)
        if rank == 0:
            q.put((t.numpy().tolist(), tp.numpy().ravel().tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('ws', [2, 3])
def test_gloo_bands_sum_to_one_process(ws):
    seed = 21
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, seed, q)) for r in range(ws)]
    for p in procs:
        p.start()
    try:
        vec, phase = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
    for p in procs:
        assert p.exitcode == 0
    slopes, flux, _, mask_idx, IF, cmd = _system(seed)
    nv = flux.size
    vec = np.array(vec, dtype=np.float32)
    assert np.array_equal(vec[:2 * nv], slopes)
    assert np.array_equal(vec[2 * nv:], flux)
    assert np.array_equal(np.array(phase, dtype=np.float32), _phase(mask_idx, IF, cmd, 0, mask_idx.size))
