"""One image split into row bands across ranks (one process per GPU).

Each rank solves the first pass of its rows (`unmix_device_rows`), the ranks
exchange their bands of the first pass (one all-gather: the refinement's
guided filter needs the whole first pass), and each rank refines its rows
against the whole-image filter (`refine_device_rows`). Every pixel's solve
reads only its own inputs and the filter is deterministic, so the banded
decomposition equals the one-GPU decomposition bit for bit; the final bands
are gathered the same way when a caller wants the whole result on every rank.

The exchange runs through torch.distributed: device tensors with the NCCL
backend, host copies with gloo. With NCCL it moves L * 4 * w * rows doubles
per rank over NVLink (160 MB in all for a 1024x1024 five-layer image).
"""
from __future__ import annotations


def row_bands(height: int, world: int) -> list[tuple[int, int]]:
    """Rows [begin, end) of each rank: as even as possible, the first
    height % world bands one row longer."""
    if world < 1 or height < 0:
        raise ValueError("row_bands needs world >= 1 and height >= 0")
    base, extra = divmod(height, world)
    bands, row = [], 0
    for r in range(world):
        rows = base + (1 if r < extra else 0)
        bands.append((row, row + rows))
        row += rows
    return bands


def gather_rows(packed, width: int, height: int, layers: int, bands, rank: int, group=None):
    """All-gather of row bands of a packed [layer][pixel][RGBA] float64 tensor
    (flat, 4 * layers * width * height values): on return every rank holds
    every band's rows (rank r contributed rows bands[r]). In place."""
    import torch
    import torch.distributed as dist
    n = width * height
    view = packed.view(layers, n, 4)
    longest = max(e - b for b, e in bands) * width
    on_device = dist.get_backend(group) == "nccl"
    b0, b1 = bands[rank]
    send = torch.zeros((layers, longest, 4), dtype=packed.dtype, device=packed.device if on_device else "cpu")
    send[:, :(b1 - b0) * width] = view[:, b0 * width:b1 * width]
    recv = [torch.empty_like(send) for _ in bands]
    dist.all_gather(recv, send, group=group)
    for r, (b, e) in enumerate(bands):
        if r != rank and e > b:
            view[:, b * width:e * width] = recv[r][:, :(e - b) * width].to(packed.device)
    return packed


def decompose(width: int, height: int, d_image, layers, d_first, d_final, rank: int, world: int, opaque=True,
              smooth=True, solver=None, d_status=None, group=None, gather_final=False, stream=None):
    """Both passes of one image resident on every rank's GPU (`d_image`:
    interleaved RGB float64 tensor), split into row bands. `d_first` /
    `d_final`: float64 device tensors of 4 * L * width * height values; on
    return `d_first` holds the whole first pass on every rank and `d_final`
    this rank's rows (every row with gather_final). Returns this rank's
    (row_begin, row_end)."""
    from . import refine_device_rows, unmix_device_rows
    import torch
    L = len(layers)
    bands = row_bands(height, world)
    b0, b1 = bands[rank]
    unmix_device_rows(width, height, d_image.data_ptr(), layers, d_first.data_ptr(), b0, b1, opaque=opaque,
                      solver=solver, d_status=d_status.data_ptr() if d_status is not None else None, stream=stream)
    torch.cuda.synchronize()
    if world > 1:
        gather_rows(d_first, width, height, L, bands, rank, group)
    refine_device_rows(width, height, d_image.data_ptr(), layers, d_first.data_ptr(), d_final.data_ptr(), b0, b1,
                       opaque=opaque, smooth=smooth, solver=solver,
                       d_status=d_status.data_ptr() if d_status is not None else None, stream=stream)
    torch.cuda.synchronize()
    if gather_final and world > 1:
        gather_rows(d_final, width, height, L, bands, rank, group)
    return b0, b1
