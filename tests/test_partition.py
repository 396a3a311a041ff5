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


def _stage_setup():
    """Couette-type quad mesh (x periodic, diffuse walls at y = -+0.5), P2,
    64 velocities, a seeded non-uniform state and the global FR oracle."""
    from oracle.fr import FROracle
    gold = os.path.join(os.path.dirname(__file__), 'golden', 'shapes_quad_p2.npz')
    g = np.load(gold)
    ops = {'M0': g['M0'], 'M132': g['M132'], 'M3': g['M3']}
    mesh = StructuredMesh((6, 3), (0.0, -0.5), (1.5, 0.5), periodic='x')
    geo = ElementGeometry(mesh, 2)
    c0 = np.linspace(-3.0, 3.0, 4)
    N = len(c0)
    idx = np.arange(N**3)
    cv = np.stack([c0[idx // (N * N)], c0[(idx // N) % N], c0[idx % N]])
    fw = np.exp(-np.sum(cv**2, axis=0))
    walls = [(np.array([-0.3, 0.0, 0.0]), fw, 'dgfs-wall-diffuse'),
             (np.array([0.3, 0.0, 0.0]), fw, 'dgfs-wall-diffuse')]
    rng = np.random.default_rng(17)
    u = fw[None, None, :] * (1.0 + 0.3 * rng.uniform(size=(geo.neles, geo.nupts, N**3)))
    return ops, geo, c0, walls, u


def _stage_worker(rank, world, port, q):
    from oracle.fr import FROracle
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        ops, geo, c0, walls, u = _stage_setup()
        mesh = StructuredMesh((6, 3), (0.0, -0.5), (1.5, 0.5), periodic='x')
        dom = LocalDomain(geo, slab_partition(mesh, world), rank)
        orc = FROracle(ops, dom, c0, 0.1, walls, bcid=dom.wall_bcid)
        ul = u[dom.elems]
        uf = orc.disu(ul)                                  # local face values
        nf, nv = dom.nfpts, ul.shape[2]

        class Part:                                        # what the transport reads
            domain = dom
            _uf_rows = torch.cat([torch.from_numpy(uf.reshape(-1, nv)),
                                  torch.full((dom.nghost, nv), float('nan'), dtype=torch.float64)])
            _send_rows = {r: torch.as_tensor(rows) for r, rows in dom.send.items()}
        tr = NCCLTransport()
        pending = tr.start(Part)                           # posted, completed later
        bc = orc.update_bc(uf)                             # work between start and wait
        tr.wait(pending)
        ghost = Part._uf_rows[dom.neles * nf:].numpy()
        dt = 1e-3
        u1 = ul + dt * orc.rhs(ul, bc=bc, ghost=ghost)
        q.put((rank, dom.elems.tolist(), u1, bool(np.isfinite(ghost).all())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('world', [2, 3])
def test_fr_stage_over_gloo_ranks_equals_single_domain(world):
    """One explicit FR stage u + dt L(u) on a slab-partitioned mesh, each rank
    a process exchanging its halo face values through NCCLTransport (gloo),
    equals the single-domain stage (FP64 oracle arithmetic)."""
    from oracle.fr import FROracle
    ops, geo, c0, walls, u = _stage_setup()
    orc = FROracle(ops, geo, c0, 0.1, walls, bcid=geo.wall_bcid)
    ref = u + 1e-3 * orc.rhs(u)
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = 29600 + (os.getpid() + 7 * world) % 1000
    procs = [ctx.Process(target=_stage_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = np.full_like(ref, np.nan)
    for rank, elems, u1, ghost_ok in res:
        assert ghost_ok
        got[elems] = u1
    assert np.isfinite(got).all()
    assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref))
    assert np.max(np.abs(ref - u)) > 1e-6                 # the stage did something
