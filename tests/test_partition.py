"""Domain decomposition host logic: local tables against the global mesh,
and the halo exchange over a 2-rank gloo process group (CPU)."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from frfs_b200.mesh import ElementGeometry, StructuredMesh
from frfs_b200.partition import LocalDomain, NCCLTransport, slab_partition


def _geo(kind='quad'):
    if kind == 'quad':
        mesh = StructuredMesh((6, 3), (0.0, -0.5), (1.5, 0.5), periodic='x')
    else:
        mesh = StructuredMesh((4, 2, 2), (0, 0, 0), (1, 1, 1), periodic='xz')
    return mesh, ElementGeometry(mesh, 2)


@pytest.mark.parametrize('kind,nparts', [('quad', 2), ('quad', 3), ('hex', 2), ('hex', 4)])
def test_local_tables_match_global(kind, nparts):
    mesh, geo = _geo(kind)
    parts = slab_partition(mesh, nparts)
    assert sorted(np.concatenate(parts).tolist()) == list(range(geo.neles))
    doms = [LocalDomain(geo, parts, r) for r in range(nparts)]
    nf = geo.nfpts
    for d in doms:
        ghost_src = {}
        for r, (row, cnt) in d.recv.items():
            send = doms[r].send[d.rank]
            assert len(send) == cnt
            for i, lrow in enumerate(send):
                ghost_src[row + i] = int(parts[r][lrow // nf]) * nf + int(lrow % nf)
        for el, e in enumerate(d.elems):
            for f in range(nf):
                g, l = int(geo.nbr[e, f]), int(d.nbr[el, f])
                if g < 0:
                    assert l < 0
                    w = -1 - l
                    assert tuple(d.wall_fpts[w]) == (el, f)
                elif l < d.neles * nf:
                    assert int(d.elems[l // nf]) * nf + l % nf == g
                else:
                    assert ghost_src[l] == g


class _FakeSystem:
    def __init__(self, dom, nv=5):
        self.domain = dom
        nf = dom.nfpts
        self._uf_rows = torch.full((dom.neles * nf + dom.nghost, nv), -1.0, dtype=torch.float64)
        for el, e in enumerate(dom.elems):
            for f in range(nf):
                self._uf_rows[el * nf + f] = float(e * nf + f)
        self._send_rows = {r: torch.as_tensor(rows) for r, rows in dom.send.items()}


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        mesh, geo = _geo('quad')
        parts = slab_partition(mesh, world)
        dom = LocalDomain(geo, parts, rank)
        sysf = _FakeSystem(dom)
        NCCLTransport().exchange(sysf)
        nf = geo.nfpts
        ok = True
        for el, e in enumerate(dom.elems):
            for f in range(nf):
                l = int(dom.nbr[el, f])
                if l >= dom.neles * nf:
                    ok &= bool((sysf._uf_rows[l] == float(geo.nbr[e, f])).all())
        q.put((rank, ok, dom.nghost))
    finally:
        dist.destroy_process_group()


def test_halo_exchange_two_ranks_gloo():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok for _, ok, _ in res)
    assert all(ng > 0 for _, _, ng in res)
