"""Row bands of one image across ranks: the band split, the all-gather of
packed [layer][pixel][RGBA] bands over gloo (two and three CPU ranks), and on
the GPU two ranks (two processes, gloo exchange through the host) whose
banded decomposition equals the one-process decomposition bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from unblending_b200.bands import row_bands


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _init(rank, world, port):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    return dist


def _run(target, world, *args, timeout=300):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q) + args) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted((q.get(timeout=timeout) for _ in range(world)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return results


def test_row_bands_cover_the_rows_once():
    for h, world in [(1, 1), (7, 2), (1024, 3), (5, 8), (0, 2)]:
        bands = row_bands(h, world)
        assert len(bands) == world and bands[0][0] == 0 and bands[-1][1] == h
        assert all(b[1] == n[0] for b, n in zip(bands, bands[1:]))
        sizes = [e - b for b, e in bands]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        row_bands(4, 0)


def _gather_worker(rank, world, port, q, w, h, L):
    import torch
    from unblending_b200.bands import gather_rows
    dist = _init(rank, world, port)
    try:
        bands = row_bands(h, world)
        n = w * h
        packed = torch.full((4 * L * n,), -1.0, dtype=torch.float64)
        v = packed.view(L, n, 4)
        b0, b1 = bands[rank]
        for l in range(L):
            v[l, b0 * w:b1 * w] = torch.arange(b0 * w, b1 * w, dtype=torch.float64)[:, None] + 1000.0 * l
        gather_rows(packed, w, h, L, bands, rank)
        q.put((rank, packed.numpy().copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,w,h,L", [(2, 5, 7, 3), (3, 4, 10, 2)])
def test_gather_rows_over_gloo(world, w, h, L):
    results = _run(_gather_worker, world, w, h, L)
    n = w * h
    expect = np.empty((L, n, 4))
    for l in range(L):
        expect[l] = (np.arange(n, dtype=np.float64) + 1000.0 * l)[:, None]
    for rank, packed in results:
        assert np.array_equal(packed.reshape(L, n, 4), expect), rank


def _gpu_worker(rank, world, port, q, solver_fp64):
    import torch
    import unblending_b200 as U
    from unblending_b200 import synthetic as syn
    from unblending_b200.bands import decompose
    torch.cuda.set_device(0)
    dist = _init(rank, world, port)
    try:
        wl = syn.workload("rgb1024_l5", 96, 72)
        L, n = len(wl.layers), wl.pixels
        d_img = torch.from_numpy(wl.image.reshape(-1)).cuda()
        first = torch.zeros(4 * L * n, dtype=torch.float64, device="cuda")
        final = torch.zeros_like(first)
        so = U.solver_options(precision=1 if solver_fp64 else 0, radius=5)
        decompose(wl.width, wl.height, d_img, wl.layers, first, final, rank, world, solver=so, gather_final=True)
        q.put((rank, first.cpu().numpy(), final.cpu().numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("fp64", [False, True])
def test_two_rank_bands_equal_one_gpu(cuda, fp64):
    import torch
    from unblending_b200 import synthetic as syn
    results = _run(_gpu_worker, 2, fp64)
    wl = syn.workload("rgb1024_l5", 96, 72)
    L, n = len(wl.layers), wl.pixels
    d_img = torch.from_numpy(wl.image.reshape(-1)).cuda()
    first = torch.empty(4 * L * n, dtype=torch.float64, device="cuda")
    final = torch.empty_like(first)
    so = cuda.solver_options(precision=1 if fp64 else 0, radius=5)
    cuda.unmix_device(wl.width, wl.height, d_img.data_ptr(), wl.layers, first.data_ptr(), solver=so)
    cuda.refine_device(wl.width, wl.height, d_img.data_ptr(), wl.layers, first.data_ptr(), final.data_ptr(),
                       smooth=True, solver=so)
    torch.cuda.synchronize()
    ref_first, ref_final = first.cpu().numpy(), final.cpu().numpy()
    for rank, f1, f2 in results:
        assert np.array_equal(f1, ref_first), rank
        assert np.array_equal(f2, ref_final), rank
