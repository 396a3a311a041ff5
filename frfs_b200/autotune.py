"""Autotuner for the collision kernel's variants.

For a set of velocity grids it times every compiled variant
(``bdgfs_vhs_tiles``: CTA size, and with it pencils per thread and register
budget) on the current device with CUDA events, on a seeded batch of
Maxwellian-plus-noise cubes, and keeps the fastest.  Results are cached in
JSON keyed by (precision, Nv, Nrho, M of every grid, SM count), in
``$BDGFS_TUNE_CACHE`` or ``frfs_b200/_lib/vhs_tune.json``.
"""
import ctypes as C
import json
import os

import torch

from . import _lib

_CACHE = os.environ.get('BDGFS_TUNE_CACHE',
                        os.path.join(os.path.dirname(os.path.abspath(__file__)), '_lib',
                                     'vhs_tune.json'))


def _key(grids, nsm):
    parts = [f"{'f64' if g.dtype == torch.float64 else 'f32'}-{g.Nv}-{g.Nrho}-{g.M}" for g in grids]
    return '|'.join(parts) + f'|sm{nsm}'


def _load():
    try:
        with open(_CACHE) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(d):
    try:
        os.makedirs(os.path.dirname(_CACHE), exist_ok=True)
        tmp = _CACHE + '.tmp'
        with open(tmp, 'w') as fh:
            json.dump(d, fh, indent=1, sort_keys=True)
        os.replace(tmp, _CACHE)
    except OSError:
        pass


def variants(grids):
    arr = (_lib.VhsGrid * len(grids))(*[g.struct for g in grids])
    n = _lib.lib().bdgfs_vhs_tiles(arr, len(grids), None, 0)
    buf = (C.c_int32 * max(n, 1))()
    _lib.lib().bdgfs_vhs_tiles(arr, len(grids), buf, n)
    return [int(buf[i]) for i in range(n)]


def tune_vhs(grids, device, reps=3, force=False, record=None):
    """Fastest tile for ``grids`` (list of scattering.VHSGrid); cached."""
    props = torch.cuda.get_device_properties(device)
    key = _key(grids, props.multi_processor_count)
    cache = _load()
    if key in cache and not force:
        tile = int(cache[key]['tile'])
        for g in grids:
            g.struct.tile = tile
        return tile
    threads = variants(grids)
    if len(threads) <= 1:
        return 0
    from .scattering import VHSCollider
    gen = torch.Generator(device=device).manual_seed(1234)
    batches = []
    for gi, g in enumerate(grids):
        n3 = g.Nv**3
        ndof = 8 * props.multi_processor_count
        c0 = g.c0.to(g.dtype)
        cx = c0.view(-1, 1, 1)
        cy = c0.view(1, -1, 1)
        cz = c0.view(1, 1, -1)
        base = torch.exp(-(cx * cx + cy * cy + cz * cz)).reshape(-1) / torch.pi**1.5
        f = base.repeat(ndof, 1) * (1 + 0.01 * torch.rand(ndof, n3, device=device,
                                                          generator=gen, dtype=g.dtype))
        batches.append((gi, f.contiguous(), torch.empty_like(f), None))
    times = []
    for t in range(len(threads)):
        for g in grids:
            g.struct.tile = t
        col = VHSCollider(grids, device)
        col(batches)                       # warm-up (sets kernel attributes)
        torch.cuda.synchronize(device)
        best = float('inf')
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            col(batches)
            b.record()
            torch.cuda.synchronize(device)
            best = min(best, a.elapsed_time(b))
        times.append(best)
        del col
    tile = int(min(range(len(times)), key=lambda i: times[i]))
    for g in grids:
        g.struct.tile = tile
    cache[key] = {'tile': tile, 'threads': threads[tile],
                  'ms': {f'tile{i}-{threads[i]}thr': times[i] for i in range(len(times))}}
    _store(cache)
    if record is not None:
        record.update(cache[key])
    return tile
