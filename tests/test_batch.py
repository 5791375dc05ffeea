"""Batches of independent cases in one context (the 64 small SA bump cases
of the mixed-precision configuration): every case keeps its own Mach number
(wcns_set_block_freestream), its own wall distance (the walls of its own
blocks) and its own wall forces (wcns_forces_blocks).

CPU: the batch's topology -- block renumbering, one case's records taken
back out, the per-case Mach numbers and sizes in their ranges.
GPU: the batched context against every case on a context of its own (the
blocks do not interact, so each block's state must agree to round-off), and
single cases against the oracle."""
import numpy as np
import pytest

from tests.helpers import compare_prim_scaled
from wcns_b200 import cases


def test_batch_topology():
    b = cases.batch_case(ncases=64, seed=0)
    assert b.nblocks == 64 and len(b.groups) == 64 and len(b.block_moo) == 64
    for (ni, nj, nk), m in zip(b.dims, b.block_moo):
        assert 17 <= ni <= 49 and 17 <= nj <= 33 and nk == 17
        assert 0.3 <= m <= 0.8
    for r in b.regions:  # every record belongs to its case's block, no interface crosses cases
        assert 1 <= r[0] <= 64
        if r[7] < 0:
            assert r[14] == r[0]
    one = cases.batch_member(b, 5)
    assert one.dims == [b.dims[5]] and one.params.moo == b.block_moo[5]
    assert np.all(one.regions[:, 0] == 1)
    p = one.prim[0][4]  # the member's free stream is its own Mach number's
    assert abs(p[10, 10, 10] - 1.0 / (1.4 * one.params.moo ** 2)) < 1e-12


def _run(case, n):
    from wcns_b200.solver import Wcns
    g = Wcns(case)
    if case.sa:
        g.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])
    g.step(n, history=False)
    return g


@pytest.mark.gpu
def test_batch_equals_separate_cases():
    b = cases.batch_case(ncases=6, seed=3)
    g = _run(b, 4)
    for q in range(6):
        one = cases.batch_member(b, q)
        h = _run(one, 4)
        nb0, _ = b.groups[q]
        np.testing.assert_array_equal(g.get("dist", nb0), h.get("dist", 1))
        for name in ("r", "u", "v", "w", "p", "qke", "vist"):
            a, c = g.get(name, nb0), h.get(name, 1)
            scale = max(float(np.max(np.abs(c))), 1e-300)
            if name in ("u", "v", "w"):
                scale = max(scale, 0.3)
            assert float(np.max(np.abs(a - c))) <= 1e-12 * scale, (q, name)
        fa, fc = g.force_blocks(nb0, nb0), h.force()
        for k in ("cfx", "cfy", "cfz"):
            assert abs(fa[k] - fc[k]) <= 1e-12 * max(abs(fc[k]), 1e-12), (q, k, fa[k], fc[k])
        h.close()


@pytest.mark.gpu
@pytest.mark.parametrize("q", [0, 4])
def test_batch_member_matches_oracle(q):
    from oracle.pyoracle import Oracle
    b = cases.batch_case(ncases=6, seed=3)
    one = cases.batch_member(b, q)
    g = _run(one, 3)
    o = Oracle(one)
    o.sa_setup(one.sa["timedt_turb"], one.sa["kmaxlim"])
    o.step(3)
    e = compare_prim_scaled(g, o)
    assert max(e.values()) <= 1e-12, e
