"""Projection stacks larger than device memory: chunked, pipelined drivers.

The reference projects a scan chunk by chunk into a ``.npy`` memmap
(src/aprict/scripts/project_cbfp.py:335-470): per chunk a new device buffer,
a blocking projection, optional Poisson noise, a device-to-host copy and the
write, one after another. Here the same work is a three-stage pipeline over
two device buffers and two pinned host buffers: while chunk k is projected on
the compute stream, chunk k-1 is copied to pinned memory on a copy stream and
chunk k-2 is written to the destination array by the host. The
backprojection driver runs the mirror image (host read -> pinned -> device
-> backprojection).

Each chunk's result is its one-call result on the same views: the projection
is bit-identical to projecting the whole scan at once; the backprojection adds
the chunks' contributions one after another.
"""

from __future__ import annotations

import numpy as np
import torch

from .cb import flatpanel as fp
from .volume import FBVolume, Volume


def _chunks(m: int, per: int) -> list[slice]:
    return [slice(a, min(a + per, m)) for a in range(0, m, per)]


def _check_geometry(pg: fp.ProjGeom) -> tuple[int, int, int]:
    if len(pg.projs_list_shape) != 1:
        msg = "only flat view lists are supported by the chunked drivers"
        raise NotImplementedError(msg)
    nu, nv = int(np.asarray(pg.nu).flat[0]), int(np.asarray(pg.nv).flat[0])
    if not (np.all(np.asarray(pg.nu) == nu) and np.all(np.asarray(pg.nv) == nv)):
        msg = "the chunked drivers need one detector size for every view"
        raise NotImplementedError(msg)
    return pg.num_projs, nu, nv


def project_to_array(
    config: fp.ConfigProject,
    volume: Volume | FBVolume,
    pg: fp.ProjGeom,
    out: np.ndarray,
    *,
    views_per_chunk: int = 64,
    photons_per_pixel: float | None = None,
    seed: int | None = None,
) -> int:
    """Project ``volume`` over ``pg`` into the host array ``out`` (M, nu, nv)
    float32 -- e.g. ``np.lib.format.open_memmap(...)`` -- chunk by chunk.

    With ``photons_per_pixel`` each chunk gets Poisson noise before it is
    written: ``-log(Poisson(I0 exp(-p)) / I0)`` (project_cbfp.py:342-359).
    Returns the number of rays whose FORBILD covered-interval list overflowed.
    """
    m, nu, nv = _check_geometry(pg)
    if out.shape != (m, nu, nv) or out.dtype != np.float32:
        msg = f"out must be a float32 array of shape {(m, nu, nv)}"
        raise ValueError(msg)
    if views_per_chunk <= 0:
        msg = "views_per_chunk must be positive"
        raise ValueError(msg)
    dev = torch.device("cuda", torch.cuda.current_device())
    per = min(views_per_chunk, m)
    dbuf = [torch.empty((per, nu, nv), dtype=torch.float32, device=dev) for _ in range(2)]
    hbuf = [torch.empty((per, nu, nv), dtype=torch.float32).pin_memory() for _ in range(2)]
    compute = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    done_copy = [torch.cuda.Event() for _ in range(2)]
    gen = torch.Generator(device=dev)
    if seed is not None:
        gen.manual_seed(seed)
    overflow = torch.zeros(1, dtype=torch.int32, device=dev)
    chunks = _chunks(m, per)
    pending: list[tuple[int, slice]] = []  # (buffer, views) copied, not yet written

    def write_oldest() -> None:
        b, sl = pending.pop(0)
        done_copy[b].synchronize()
        out[sl] = hbuf[b][: sl.stop - sl.start].numpy()

    for k, sl in enumerate(chunks):
        b = k % 2
        if len(pending) == 2:
            write_oldest()  # frees buffer b
        n = sl.stop - sl.start
        d = dbuf[b][:n]
        compute.wait_event(done_copy[b])  # the previous copy out of d has finished
        d.zero_()
        ps = fp.ProjectionSet(pg.sliced(sl), data=d)
        ps._out_of_mem_counter = overflow  # noqa: SLF001  one counter for the whole scan
        fp.project(config, volume, ps)
        if photons_per_pixel is not None:
            lam = photons_per_pixel * torch.exp(-d.double())
            counts = torch.poisson(lam, generator=gen).clamp_(min=1.0)
            d.copy_(-torch.log(counts / photons_per_pixel))
        ready = torch.cuda.Event()
        ready.record(compute)
        with torch.cuda.stream(copy):
            copy.wait_event(ready)
            hbuf[b][:n].copy_(d, non_blocking=True)
            done_copy[b].record(copy)
        pending.append((b, sl))
    while pending:
        write_oldest()
    torch.cuda.synchronize()
    return int(overflow.item())


def backproject_from_array(
    config: fp.ConfigBackproject,
    volume: Volume,
    pg: fp.ProjGeom,
    projs: np.ndarray,
    *,
    views_per_chunk: int = 64,
    summand_multiplier: Volume | None = None,
) -> Volume:
    """``volume += BP(projs)`` for host projections ``projs`` (M, nu, nv)
    float32 (e.g. a ``.npy`` memmap), reading, uploading and backprojecting
    chunk by chunk with the three stages overlapped."""
    m, nu, nv = _check_geometry(pg)
    if projs.shape != (m, nu, nv) or projs.dtype != np.float32:
        msg = f"projs must be a float32 array of shape {(m, nu, nv)}"
        raise ValueError(msg)
    if views_per_chunk <= 0:
        msg = "views_per_chunk must be positive"
        raise ValueError(msg)
    dev = torch.device("cuda", torch.cuda.current_device())
    per = min(views_per_chunk, m)
    dbuf = [torch.empty((per, nu, nv), dtype=torch.float32, device=dev) for _ in range(2)]
    hbuf = [torch.empty((per, nu, nv), dtype=torch.float32).pin_memory() for _ in range(2)]
    compute = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    uploaded = [torch.cuda.Event() for _ in range(2)]
    consumed = [torch.cuda.Event() for _ in range(2)]
    chunks = _chunks(m, per)

    def stage(k: int) -> None:  # host read into pinned memory, then upload
        b, sl = k % 2, chunks[k]
        n = sl.stop - sl.start
        consumed[b].synchronize()  # the backprojection that read dbuf[b] (and hbuf[b]'s upload) is done
        hbuf[b][:n].numpy()[...] = projs[sl]
        with torch.cuda.stream(copy):
            copy.wait_event(consumed[b])
            dbuf[b][:n].copy_(hbuf[b][:n], non_blocking=True)
            uploaded[b].record(copy)

    for e in consumed:
        e.record(compute)
    if chunks:
        stage(0)
    for k, sl in enumerate(chunks):
        b = k % 2
        compute.wait_event(uploaded[b])
        n = sl.stop - sl.start
        fp.backproject(config, volume, fp.ProjectionSet(pg.sliced(sl), data=dbuf[b][:n]),
                       summand_multiplier=summand_multiplier)
        consumed[b].record(compute)
        if k + 1 < len(chunks):
            stage(k + 1)  # the host reads the next chunk while this one is backprojected
    torch.cuda.synchronize()
    return volume


__all__ = ["backproject_from_array", "project_to_array"]
