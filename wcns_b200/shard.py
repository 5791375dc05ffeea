"""Block sharding across ranks: each rank advances the blocks it owns.

The reference runs one MPI rank per group of blocks and exchanges interface
data three times per step (`exchange_bc`, `communicate_dq_npp`,
`communicate_pv_npp`, parallel.f90:1559-1674, 3020-3326).  Here every rank
holds a context (a GPU `Wcns`) of its owned blocks plus
*proxy* copies of every block within three interface hops of them, so that
each averaging set that touches an owned point -- two blocks across a face,
four along an edge, eight at a corner -- is complete in the rank's own
context.  Two exchanges per step keep the proxies equal to their owners:

  E1  before the boundary conditions: every proxy's whole ghosted state
      (r, u, v, w, p, T) from its owner;
  E3  after the update, before the prim averaging: every proxy's updated
      state from its owner.

Between them the rank runs the reference's phases on all of its blocks.  An
owned block's ghosts are copied from present blocks whose interiors are the
owners' (E1); its dq depends on its own state only, and the dq averaging
sets of its points are complete with the proxies' dq computed from the same
state; its LU-SGS is per block (block-Jacobi); its prim averaging reads the
proxies' states of E3.  A proxy's own results (its regions towards absent
blocks are dropped, so its LU-SGS sees other face values) never reach an
owned block, since E1 and E3 overwrite them first; the one local dependence
-- the residual of a proxy point near the face shared with an owned block
reading the proxy's ghosts towards an absent block -- needs the two faces
to be at least seven points apart, which `rank_case` checks.

With the Spalart-Allmaras model the state also carries qke and vist, the
model step runs as its own phase, and a third exchange (E2) refreshes the
proxies' qke and vist after it, before the viscous flux; the wall distance
of every block is the whole case's (`set_distance`), not the distance to
the walls a rank happens to hold.  The exchange moves whole
blocks, either through host arrays (`DistTransport` over torch.distributed,
`LocalTransport` between contexts of one process) or on the device: the
contexts' field slices are wrapped as CUDA tensors (wcns_field_device_ptr)
and broadcast in place over NCCL (`DeviceTransport`), or copied device to
device between the contexts of one process (`run_local(..., device=True)`).
Packing only the three-layer halos and interface faces would cut the bytes
further.
"""
from __future__ import annotations

import heapq

import numpy as np

from .cases import Case, Params

PRIM6 = ("r", "u", "v", "w", "p", "t")
SA2 = ("qke", "vist")


def lpt_partition(dims, nranks):
    """Longest-processing-time packing of blocks onto ranks by points:
    owners[b] for block b+1, blocks taken largest first onto the least
    loaded rank (ties to the lower rank)."""
    npts = [int(a) * int(b) * int(c) for a, b, c in dims]
    order = sorted(range(len(dims)), key=lambda b: (-npts[b], b))
    heap = [(0, r) for r in range(nranks)]
    owners = [0] * len(dims)
    for b in order:
        load, r = heapq.heappop(heap)
        owners[b] = r
        heapq.heappush(heap, (load + npts[b], r))
    return owners


def neighbours(case):
    """Interface partners of every block (1-based), from the BC records."""
    nb = {b: set() for b in range(1, case.nblocks + 1)}
    for r in case.regions:
        if r[7] < 0 and r[14] != r[0]:
            nb[int(r[0])].add(int(r[14]))
    return nb


def local_blocks(case, owners, rank, hops=3):
    owned = [b for b in range(1, case.nblocks + 1) if owners[b - 1] == rank]
    nbr = neighbours(case)
    local, frontier = set(owned), set(owned)
    for _ in range(hops):
        frontier = {p for b in frontier for p in nbr[b]} - local
        local |= frontier
    return owned, sorted(local)


def rank_case(case: Case, owners, rank, hops=3):
    """The rank's case: owned and proxy blocks renumbered 1..n in global
    order, with the BC records of those blocks; an interface record whose
    partner is absent is dropped (a proxy's ghosts there keep the owner's
    values), and the partner-region indices (ibcwin) are renumbered.
    Returns (case, local->global block numbers, owned mask)."""
    owned, local = local_blocks(case, owners, rank, hops)
    gmap = {g: i + 1 for i, g in enumerate(local)}
    regs_of = {b: [r for r in case.regions if int(r[0]) == b] for b in local}
    keep = {b: [int(r[7]) >= 0 or int(r[14]) in gmap for r in regs_of[b]] for b in local}
    for b in owned:
        if not all(keep[b]):
            raise ValueError(f"block {b}: an interface partner lies outside the rank's blocks")
    nbr = neighbours(case)
    for b in local:
        if b in owned:
            continue
        dropped = any(not k for k in keep[b])
        if dropped and min(case.dims[b - 1]) < 7 and any(p in owned for p in nbr[b]):
            raise ValueError(f"proxy block {b} is thinner than 7 points next to an owned block")
    rows = []
    for b in local:
        for r, k in zip(regs_of[b], keep[b]):
            if not k:
                continue
            r = np.array(r, dtype=np.int32)
            r[0] = gmap[b]
            if r[7] < 0:
                p = int(r[14])
                pos = int(r[15])  # 1-based position of the partner region in block p's list
                r[15] = 1 + sum(1 for kk in keep[p][:pos - 1] if kk)
                r[14] = gmap[p]
            rows.append(r)
    prm = Params(**{k: getattr(case.params, k) for k in Params.__dataclass_fields__})
    sub = Case(f"{case.name}_rank{rank}", prm, [case.dims[b - 1] for b in local], [case.xyz[b - 1] for b in local],
               np.array(rows, dtype=np.int32), [case.prim[b - 1] for b in local], case.nsteps,
               f"rank {rank}: owned {owned}, proxies {[b for b in local if b not in owned]}", sa=case.sa)
    return sub, local, [b in owned for b in local]


# --------------------------------------------------------------------------
# transports: how a block's state reaches the ranks that hold it as a proxy

class LocalTransport:
    """All ranks in one process (their contexts advanced in turn)."""

    def __init__(self):
        self.store = {}

    def share(self, block, owner, rank, arrays):
        if rank == owner:
            self.store[block] = [a.copy() for a in arrays]
            return arrays
        return self.store[block]


class DistTransport:
    """torch.distributed (gloo or a gloo group beside NCCL): one broadcast
    of the block's six arrays from its owner."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group

    def share(self, block, owner, rank, arrays_or_shapes):
        import torch
        out = []
        for a in arrays_or_shapes:
            t = torch.from_numpy(np.ascontiguousarray(a)) if rank == owner else torch.empty(a, dtype=torch.float64)
            self.dist.broadcast(t, src=owner, group=self.group)
            out.append(t.numpy())
        return out


class DeviceTransport:
    """torch.distributed over NCCL on the contexts' own device memory: each
    array of a shared block is broadcast from its owner's field slice
    straight into the proxies' slices (a rank that does not hold the block
    receives into scratch)."""

    device = True

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group

    def share(self, block, owner, rank, tensors):
        for t in tensors:
            self.dist.broadcast(t, src=owner, group=self.group)
        return tensors


# --------------------------------------------------------------------------
# a backend runs the reference's phases on a rank's case: GpuBackend here
# (the tests add one over the CPU oracle, which is their checker)

class GpuBackend:
    def __init__(self, case, flags=0):
        from .solver import Wcns
        self.g = Wcns(case, flags=flags)
        self.sa = case.sa is not None
        if self.sa:
            self.g.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])

    def phase(self, name):
        getattr(self.g, {"boundary_all": "boundary_all", "initial_q_dq_c_t": "initial_q_dq_c_t",
                         "timestep": "timestep_tgh", "rhs_vis": "r_h_s_vis", "rhs_vis_flux": "r_h_s_vis_flux",
                         "turbulence": "turbulence", "communicate_dq": "communicate_dq_npp",
                         "rhs_invis": "r_h_s_invis", "lhs": "l_h_s_tgh", "communicate_pv": "communicate_pv_npp"}[name])()

    def get_state(self, nb, fields=None):
        """The ghosted arrays of `fields` (default: r,u,v,w,p,T and, with the
        SA model, qke and vist)."""
        if fields is None:
            out = list(self.g.get_prim(nb))
            return out + [self.g.get(n, nb) for n in SA2] if self.sa else out
        return [self.g.get(n, nb) for n in fields]

    def set_state(self, nb, arrays, fields=None):
        if fields is None:
            self.g.set_prim(nb, arrays[:6])
            for n, a in zip(SA2 if self.sa else (), arrays[6:]):
                self.g.set(n, nb, a)
            return
        for n, a in zip(fields, arrays):
            self.g.set(n, nb, a)

    def set_field(self, name, nb, arr):
        self.g.set(name, nb, arr)

    def device_views(self, nb, fields):
        """CUDA tensors aliasing block nb's slices of `fields`."""
        import torch
        return [torch.as_tensor(self.g.device_view(n, nb), device="cuda") for n in fields]

    def sync(self):
        self.g.sync()

    def residual(self):
        res, rmax, _ = self.g.residual_curve()
        return res, rmax

    def get(self, name, nb):
        return self.g.get(name, nb)


class ShardedRank:
    """One rank of a block-sharded run."""

    def __init__(self, case: Case, owners, rank, backend, transport):
        self.case, self.owners, self.rank = case, list(owners), rank
        self.sub, self.local, self.owned_mask = rank_case(case, owners, rank)
        self.lmap = {g: i + 1 for i, g in enumerate(self.local)}
        self.be = backend(self.sub) if callable(backend) else backend
        self.tr = transport
        self.sa = case.sa is not None
        # every block held as a proxy somewhere: the exchanges walk these in
        # global order on every rank (the same collective sequence everywhere)
        self.shared = sorted({b for r in range(max(self.owners) + 1)
                              for b in local_blocks(case, self.owners, r)[1] if self.owners[b - 1] != r})

    def fields(self, which):
        """The exchanged arrays: the whole state (E1, E3) or qke and vist (E2)."""
        if which == "sa":
            return SA2
        return PRIM6 + (SA2 if self.sa else ())

    def set_distance(self, dist):
        """The wall distance of every local block from {global block: ghosted
        array} of the whole case (after the backend's SA set-up)."""
        for g, nb in self.lmap.items():
            self.be.set_field("dist", nb, dist[g])

    def _exchange(self, which="state"):
        """One exchange over a DistTransport or a DeviceTransport: every
        shared block broadcast from its owner, in global block order on
        every rank."""
        names = self.fields(which)
        if getattr(self.tr, "device", False):
            import torch
            self.be.sync()
            torch.cuda.synchronize()
            for b in self.shared:
                ni, nj, nk = self.case.dims[b - 1]
                ts = (self.be.device_views(self.lmap[b], names) if b in self.lmap else
                      [torch.empty((nk + 6, nj + 6, ni + 6), dtype=torch.float64, device="cuda") for _ in names])
                self.tr.share(b, self.owners[b - 1], self.rank, ts)
            torch.cuda.synchronize()
            return
        for b in self.shared:
            owner = self.owners[b - 1]
            ni, nj, nk = self.case.dims[b - 1]
            arrays = (self.be.get_state(self.lmap[b], names) if self.rank == owner
                      else [(nk + 6, nj + 6, ni + 6)] * len(names))
            got = self.tr.share(b, owner, self.rank, arrays)
            if self.rank != owner and b in self.lmap:
                self.be.set_state(self.lmap[b], got, names)

    def publish(self, store, which="state"):
        """LocalTransport: the arrays of the owned blocks others hold."""
        names = self.fields(which)
        for b in self.shared:
            if self.owners[b - 1] == self.rank:
                store[b] = [a.copy() for a in self.be.get_state(self.lmap[b], names)]

    def pull(self, store, which="state"):
        """LocalTransport: every proxy's arrays from the store."""
        names = self.fields(which)
        for b in self.shared:
            if self.owners[b - 1] != self.rank and b in self.lmap:
                self.be.set_state(self.lmap[b], store[b], names)

    def phases_to_model(self):
        """From the BCs to the SA model step (E1 before it)."""
        for name in ("boundary_all", "initial_q_dq_c_t", "timestep"):
            self.be.phase(name)
        if self.sa:
            self.be.phase("turbulence")

    def phases_to_update(self):
        """From the viscous flux to the update (E2 before it with the SA model)."""
        if self.case.params.nvis == 1:
            self.be.phase("rhs_vis_flux" if self.sa else "rhs_vis")
            self.be.phase("communicate_dq")
        self.be.phase("rhs_invis")
        self.be.phase("communicate_dq")
        self.be.phase("lhs")

    def finish_after_e3(self):
        """Prim averaging and the owned blocks' residual means."""
        self.be.phase("communicate_pv")
        res, _ = self.be.residual()
        out = {}
        for i, g in enumerate(self.local):
            if self.owned_mask[i]:
                ni, nj, nk = self.case.dims[g - 1]
                out[g] = (float(res[i]), (ni - 2) * (nj - 2) * (nk - 2) * 5)
        return out

    def step(self, nsteps=1):
        """nsteps whole steps over a DistTransport (every rank calls it):
        E1, the phases to the model step, E2 (SA), the phases to the update,
        E3, the prim averaging; the residual RMS of every step from an
        all-reduce of the block sums."""
        import torch
        hist = []
        for _ in range(nsteps):
            self._exchange()  # E1
            self.phases_to_model()
            if self.sa:
                self._exchange("sa")  # E2
            self.phases_to_update()
            self._exchange()  # E3
            mine = self.finish_after_e3()
            t = torch.tensor([sum(m * n for m, n in mine.values()), float(sum(n for _, n in mine.values()))],
                             dtype=torch.float64)
            self.tr.dist.all_reduce(t, group=self.tr.group)
            hist.append(float(np.sqrt(t[0].item() / t[1].item())))
        return np.array(hist)

    def get(self, name, global_nb):
        return self.be.get(name, self.lmap[global_nb])


def rms_of(block_res):
    """The residual RMS of residual_curve from the per-block means of all
    ranks ({block: (mean, points)}), summed in block order."""
    total = npts = 0
    for b in sorted(block_res):
        m, n = block_res[b]
        total += m * n
        npts += n
    return float(np.sqrt(total / npts))


def run_local(case, nranks, nsteps, backend, owners=None, dist=None, device=False):
    """All ranks in one process, in turn: each step every rank publishes its
    owned states, pulls its proxies (E1) and runs to the model step; with
    the SA model the ranks then exchange qke and vist (E2); every rank runs
    to the update, publishes its updated states, pulls (E3), averages prim
    and reports its residual means.  `dist` ({global block: ghosted array})
    sets the whole case's wall distance.  Returns the ranks and the
    residual RMS of every step."""
    owners = list(owners) if owners is not None else lpt_partition(case.dims, nranks)
    tr = LocalTransport()
    ranks = [ShardedRank(case, owners, r, backend, tr) for r in range(nranks)]
    if dist is not None:
        for rk in ranks:
            rk.set_distance(dist)

    def exchange(which):
        if device:  # device-to-device copies from the owners' slices into the proxies'
            import torch
            for rk in ranks:
                rk.be.sync()
            torch.cuda.synchronize()
            names = ranks[0].fields(which)
            for rk in ranks:
                for b in rk.shared:
                    own = ranks[owners[b - 1]]
                    if own is rk or b not in rk.lmap:
                        continue
                    for dst, src in zip(rk.be.device_views(rk.lmap[b], names), own.be.device_views(own.lmap[b], names)):
                        dst.copy_(src)
            torch.cuda.synchronize()
            return
        for rk in ranks:
            rk.publish(tr.store, which)
        for rk in ranks:
            rk.pull(tr.store, which)

    hist = []
    for _ in range(nsteps):
        exchange("state")
        for rk in ranks:
            rk.phases_to_model()
        if case.sa is not None:
            exchange("sa")
        for rk in ranks:
            rk.phases_to_update()
        exchange("state")
        res = {}
        for rk in ranks:
            res.update(rk.finish_after_e3())
        hist.append(rms_of(res))
    return ranks, np.array(hist)
