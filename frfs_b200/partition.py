"""Domain decomposition of the FR advection and the halo exchange.

Counterpart of the reference's multi-rank path: METIS element partitions
(frfs/partitioners/metis.py:117-183), MPI interfaces that pack face values,
send/receive them and run the one-sided flux (frfs/solvers/dgfs/inters.py:
61-112, frfs/backends/base/packing.py:9-39).  Here:

* elements are split into contiguous slabs along the longest mesh axis
  (structured meshes; every rank gets whole elements and all their DOFs, so
  the collision operator needs no communication);
* a face point whose neighbour lives on another rank gets a ghost row
  appended after the local face values ``uf[E_local * nfpts + slot]``; the
  local neighbour table points at it, so the fused FR kernel runs unchanged;
* after ``disu`` each rank sends the face rows its neighbours need and
  receives its ghost rows (``NCCLTransport``: torch.distributed batched
  send/recv, NCCL on GPUs, gloo on CPUs; ``LocalTransport``: device copies
  between virtual ranks of one process).
"""
import numpy as np
import torch


def slab_partition(mesh, nparts):
    """Element ids of each part: contiguous slabs along the longest axis."""
    ax = int(np.argmax(mesh.shape))
    n = mesh.shape[ax]
    if nparts > n:
        raise ValueError(f'{nparts} parts for {n} element layers')
    bounds = np.linspace(0, n, nparts + 1).round().astype(int)
    coord = np.array([c[ax] for c in mesh.cells])
    return [np.nonzero((coord >= bounds[p]) & (coord < bounds[p + 1]))[0] for p in range(nparts)]


class LocalDomain:
    """Local view of a global ElementGeometry for one part.

    Attributes: ``elems`` (global ids), local ``smats``/``rcpdjac``/normals,
    ``nbr`` with ghost slots, ``wall_fpts``/``wall_bcid`` (local),
    ``recv[r] = (first ghost row, count)`` and ``send[r]`` (local face rows
    to pack for rank r, in the order rank r expects them).
    """

    def __init__(self, geo, parts, rank):
        self.rank, self.nparts = rank, len(parts)
        self.geo = geo
        elems = np.asarray(parts[rank])
        owner = np.empty(geo.neles, dtype=np.int64)
        lid = np.empty(geo.neles, dtype=np.int64)
        for p, es in enumerate(parts):
            owner[es] = p
            lid[es] = np.arange(len(es))
        nf = geo.nfpts
        E = len(elems)
        self.elems, self.neles, self.nfpts = elems, E, nf
        self.ndims, self.nupts = geo.ndims, geo.nupts
        self.shape = geo.shape
        self.smats = geo.smats[elems]
        self.rcpdjac = geo.rcpdjac[elems]
        self.djac = geo.djac[elems]
        self.norm_pnorm = geo.norm_pnorm[elems]
        self.mag_pnorm = geo.mag_pnorm[elems]
        self.plocupts = geo.plocupts[elems]
        self.plocfpts = geo.plocfpts[elems]
        # ghost slots, grouped by the owning rank (so each receive is one block)
        need = {}                                    # rank -> list of global fpt ids
        for el, e in enumerate(elems):
            for f in range(nf):
                nb = int(geo.nbr[e, f])
                if nb >= 0 and owner[nb // nf] != rank:
                    need.setdefault(int(owner[nb // nf]), []).append(nb)
        self.recv, slot_of = {}, {}
        row = E * nf
        for r in sorted(need):
            ids = sorted(set(need[r]))
            self.recv[r] = (row, len(ids))
            for i, g in enumerate(ids):
                slot_of[g] = row + i
            row += len(ids)
        self.nghost = row - E * nf
        nbr = np.empty((E, nf), dtype=np.int64)
        for el, e in enumerate(elems):
            for f in range(nf):
                nb = int(geo.nbr[e, f])
                if nb < 0:
                    nbr[el, f] = nb                   # wall: remapped below
                elif owner[nb // nf] == rank:
                    nbr[el, f] = lid[nb // nf] * nf + nb % nf
                else:
                    nbr[el, f] = slot_of[nb]
        # local walls
        wf, wb = [], []
        for el, e in enumerate(elems):
            for f in range(nf):
                nb = int(geo.nbr[e, f])
                if nb < 0:
                    w = -1 - nb
                    nbr[el, f] = -1 - len(wf)
                    wf.append((el, f))
                    wb.append(int(geo.wall_bcid[w]))
        self.nbr = nbr.astype(np.int32)
        self.wall_fpts = np.array(wf, dtype=np.int64).reshape(-1, 2)
        self.wall_bcid = np.array(wb, dtype=np.int64)
        self.wall_names = geo.wall_names
        # what every other rank needs from me (same sorted order as its recv)
        self.send = {}
        for r in range(self.nparts):
            if r == rank:
                continue
            other = np.asarray(parts[r])
            ids = set()
            for e in other:
                for f in range(nf):
                    nb = int(geo.nbr[e, f])
                    if nb >= 0 and owner[nb // nf] == rank:
                        ids.add(nb)
            if ids:
                self.send[r] = np.array([lid[g // nf] * nf + g % nf for g in sorted(ids)],
                                        dtype=np.int64)


class LocalTransport:
    """Halo exchange between virtual ranks of one process (device copies)."""

    def __init__(self, systems):
        self.systems = systems

    def exchange(self, system):
        rank = system.domain.rank
        for r, (row, cnt) in system.domain.recv.items():
            src = self.systems[r]
            rows = src._send_rows[rank]
            system._uf_rows[row:row + cnt].copy_(src._uf_rows.index_select(0, rows))


def step_rk2_virtual(systems, dt):
    """One dgfs-tvd-rk2 step of virtual ranks sharing one process (stage by
    stage across all parts, so every exchange sees its neighbours' disu)."""
    for s in systems:
        s.collide(0.0, 0, 1)
        s.advect_begin(0, 1)
    for s in systems:
        s.advect_end(0.0, 1.0, dt, x1=1, c1=dt)
    for s in systems:
        s.collide(dt, 1, 2)
        s.advect_begin(1, 0)
    for s in systems:
        s.advect_end(dt, 0.5, 0.5 * dt, x1=2, c1=0.5 * dt, x2=0, c2=0.5)


def bind_local_transports_bi(systems):
    """Virtual ranks of the 'dgfsbi' system in one process: species p of
    every rank exchanges with species p of its neighbours."""
    for p in range(systems[0].nspcs()):
        tr = LocalTransport([b.species[p] for b in systems])
        for b in systems:
            b.species[p].transport = tr


def step_rk2_virtual_bi(systems, dt):
    """One dgfsbi-tvd-rk2 step of virtual ranks sharing one process."""
    for b in systems:
        b.collide_banks(0.0, 0, 1)
        for sp in b.species:
            sp.advect_begin(0, 1)
    for b in systems:
        for sp in b.species:
            sp.advect_end(0.0, 1.0, dt, x1=1, c1=dt)
    for b in systems:
        b.collide_banks(dt, 1, 2)
        for sp in b.species:
            sp.advect_begin(1, 0)
    for b in systems:
        for sp in b.species:
            sp.advect_end(dt, 0.5, 0.5 * dt, x1=2, c1=0.5 * dt, x2=0, c2=0.5)


class NCCLTransport:
    """Halo exchange between processes: one batched send/recv per neighbour
    (torch.distributed; NCCL for CUDA tensors, gloo for CPU tensors).

    ``start`` posts the exchange and returns at once; ``wait`` completes
    it.  With NCCL the transfers run on NCCL's stream after the work already
    queued on the current stream (the face values), and ``wait`` makes the
    current stream wait for them, so device work queued between the two
    calls (the collision launch, which does not read face values) overlaps
    the transfer.  As the reference's two queues do (solvers/dgfs/system.py:
    151-166), the exchange is hidden behind interior work."""

    def __init__(self, group=None):
        self.group = group

    def start(self, system):
        import torch.distributed as dist
        ops = []
        bufs = []
        for r, rows in sorted(system._send_rows.items()):
            b = system._uf_rows.index_select(0, rows)
            bufs.append(b)
            ops.append(dist.P2POp(dist.isend, b, r, group=self.group))
        for r, (row, cnt) in sorted(system.domain.recv.items()):
            ops.append(dist.P2POp(dist.irecv, system._uf_rows[row:row + cnt], r,
                                  group=self.group))
        reqs = dist.batch_isend_irecv(ops) if ops else []
        return reqs, bufs                        # the send buffers live until wait

    @staticmethod
    def wait(pending):
        reqs, _ = pending
        for req in reqs:
            req.wait()

    def exchange(self, system):
        self.wait(self.start(system))
