"""Block sharding (wcns_b200/shard.py): ranks own blocks, hold proxies of
the blocks within three interface hops, and refresh them from their owners
before the BCs (E1) and after the update (E3).

CPU: the LPT partition; the ranks' BC records (partners and partner-region
indices point back, absent partners dropped); the sharded run on the oracle
-- ranks in one process, and two gloo ranks exchanging through
torch.distributed -- against the single-process oracle.
GPU: the sharded run on GPU contexts against one GPU context."""
import os
import socket
import sys

import numpy as np
import pytest

from tests.helpers import interior
from wcns_b200 import cases, shard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class OracleBackend:
    """The phases of a rank's case on the CPU oracle (the checker)."""

    def __init__(self, case):
        from oracle.pyoracle import Oracle
        self.o = Oracle(case)
        self.sa = case.sa is not None
        if self.sa:
            self.o.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"], distance=False)

    def phase(self, name):
        self.o.phase(name)

    def get_state(self, nb, fields=None):
        names = fields or (shard.PRIM6 + (shard.SA2 if self.sa else ()))
        return [self.o.get(n, nb) for n in names]

    def set_state(self, nb, arrays, fields=None):
        if fields is None:
            self.o.set_prim(nb, arrays[:6])
            for n, a in zip(shard.SA2 if self.sa else (), arrays[6:]):
                self.o.set(n, nb, a)
            return
        for n, a in zip(fields, arrays):
            self.o.set(n, nb, a)

    def set_field(self, name, nb, arr):
        self.o.set(name, nb, arr)

    def residual(self):
        res, rmax, _ = self.o.residual()
        return res, rmax

    def get(self, name, nb):
        return self.o.get(name, nb)


def laminar_channel():
    """A 32-block laminar channel (8 x 2 x 2 blocks) with its bump."""
    c = cases.channel_case(ni=97, nj=25, nk=17, bx=8, by=2, bz=2, first=1.0e-3)
    c.sa = None
    c.params.nvis = 1
    return c


def sa_channel():
    """The same 32 blocks with the Spalart-Allmaras model."""
    return cases.channel_case(ni=97, nj=25, nk=17, bx=8, by=2, bz=2, first=1.0e-3)


def full_distance(case):
    """The whole case's wall distance per block (the oracle's exact minimum)."""
    from oracle.pyoracle import Oracle
    o = Oracle(case)
    o.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])
    return {g: o.get("dist", g) for g in range(1, case.nblocks + 1)}


def slabs(case, nranks):
    """Owners by the block's x position: contiguous slabs of block columns."""
    xs = [round(float(x[0].min()), 6) for x in case.xyz]
    cols = sorted(set(xs))
    per = -(-len(cols) // nranks)
    return [cols.index(v) // per for v in xs]


def test_lpt_partition_balances_points():
    dims = cases.plate_case().dims
    for n in (2, 3, 4):
        owners = shard.lpt_partition(dims, n)
        assert sorted(set(owners)) == list(range(n))
        loads = [sum(a * b * c for (a, b, c), o in zip(dims, owners) if o == r) for r in range(n)]
        assert max(loads) - min(loads) <= max(a * b * c for a, b, c in dims)
        assert owners == shard.lpt_partition(dims, n)


def test_rank_case_records_point_back():
    c = laminar_channel()
    owners = slabs(c, 2)
    for rank in range(2):
        sub, local, owned = shard.rank_case(c, owners, rank)
        assert sum(owned) == 16 and len(local) == 28
        per = {b: [r for r in sub.regions if r[0] == b] for b in range(1, len(local) + 1)}
        for b, regs in per.items():
            for r in regs:
                if r[7] < 0:
                    q = per[int(r[14])][int(r[15]) - 1]
                    assert q[7] < 0 and int(q[14]) == b and per[b][int(q[15]) - 1] is r
        # owned blocks keep every record; proxies next to the absent columns lose some
        for i, g in enumerate(local):
            full = int(np.sum(c.regions[:, 0] == g))
            if owned[i]:
                assert len(per[i + 1]) == full
    # a proxy thinner than 7 points that loses regions next to an owned block
    thin = cases.channel_case(ni=33, nj=25, nk=17, bx=8, by=2, bz=2, first=1.0e-3)
    thin.sa = None
    with pytest.raises(ValueError):
        shard.rank_case(thin, slabs(thin, 2), 0, hops=1)


def _single(case, n):
    from oracle.pyoracle import Oracle
    o = Oracle(case)
    if case.sa:
        o.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])
    h = o.step(n)
    return o, h


def _compare(case, ranks, ref, owners):
    worst = 0.0
    for rk in ranks:
        for g in range(1, case.nblocks + 1):
            if owners[g - 1] != rk.rank:
                continue
            d = case.dims[g - 1]
            for n in ("r", "u", "v", "w", "p") + (("qke", "vist") if case.sa else ()):
                a, b = interior(rk.get(n, g), d), interior(ref.get(n, g), d)
                worst = max(worst, float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 0.3))
    return worst


@pytest.mark.parametrize("which", ["plate_lpt", "channel_slabs", "sa_channel_slabs"])
def test_sharded_oracle_in_one_process_matches_single(which):
    case = {"plate_lpt": cases.small_plate_case, "channel_slabs": laminar_channel, "sa_channel_slabs": sa_channel}[which]()
    owners = shard.lpt_partition(case.dims, 2) if which == "plate_lpt" else slabs(case, 2)
    n = 4
    dist = full_distance(case) if case.sa else None
    ranks, hist = shard.run_local(case, 2, n, OracleBackend, owners=owners, dist=dist)
    ref, href = _single(case, n)
    worst = _compare(case, ranks, ref, owners)
    print(f"{which}: owned blocks vs single oracle, max rel {worst:.2e}; rms {hist[-1]:.6e} vs {href[-1]:.6e}")
    assert worst <= 1e-13
    np.testing.assert_allclose(hist, href, rtol=1e-12)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, nsteps, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from tests.test_shard import OracleBackend, laminar_channel, slabs
    from wcns_b200 import shard as sh
    dist.init_process_group("gloo", rank=rank, world_size=world)
    case = laminar_channel()
    owners = slabs(case, world)
    rk = sh.ShardedRank(case, owners, rank, OracleBackend, sh.DistTransport())
    hist = rk.step(nsteps)
    mine = {g: [rk.get(n, g) for n in ("r", "u", "v", "w", "p")] for g in range(1, case.nblocks + 1)
            if owners[g - 1] == rank}
    out.put((rank, hist, mine))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks_exchange_matches_single():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port, n = _free_port(), 3
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=600) for _ in range(2)]
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    case = laminar_channel()
    ref, href = _single(case, n)
    worst = 0.0
    for rank, hist, mine in got:
        np.testing.assert_allclose(hist, href, rtol=1e-12)
        for g, arrs in mine.items():
            d = case.dims[g - 1]
            for a, name in zip(arrs, ("r", "u", "v", "w", "p")):
                b = interior(ref.get(name, g), d)
                worst = max(worst, float(np.max(np.abs(interior(a, d) - b))) / max(float(np.max(np.abs(b))), 0.3))
    print(f"two gloo ranks: owned blocks vs single oracle, max rel {worst:.2e}")
    assert worst <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("device", [False, True])
@pytest.mark.parametrize("which", ["plate_lpt", "channel_slabs", "sa_channel_slabs"])
def test_sharded_gpu_contexts_match_one_context(which, device):
    from wcns_b200.solver import Wcns
    case = {"plate_lpt": cases.small_plate_case, "channel_slabs": laminar_channel, "sa_channel_slabs": sa_channel}[which]()
    owners = shard.lpt_partition(case.dims, 2) if which == "plate_lpt" else slabs(case, 2)
    n = 4
    ref = Wcns(case)
    dist = None
    if case.sa:
        ref.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])
        dist = {g: ref.get("dist", g) for g in range(1, case.nblocks + 1)}
    ranks, hist = shard.run_local(case, 2, n, shard.GpuBackend, owners=owners, dist=dist, device=device)
    href = ref.step(n)
    worst = _compare(case, ranks, ref, owners)
    print(f"{which} on the GPU ({'device' if device else 'host'} exchange): owned blocks vs one context, max rel {worst:.2e}")
    assert worst <= 1e-13
    np.testing.assert_allclose(hist, href, rtol=1e-12)
