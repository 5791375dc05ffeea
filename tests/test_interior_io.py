"""wcns_set_interior / wcns_get_interior: the interior points of named fields
of every block in the flow-file layout, through the context's contiguous
staging buffer (one copy per block and field, a scatter or gather kernel
per field).  Checked against the per-block ghosted transfers (wcns_get_field
/ wcns_set_field): values, untouched ghosts, blocks skipped with a null
array, the SA model's fields, and a second call with more fields (the
staging buffer grows)."""
import numpy as np
import pytest

from tests.helpers import interior
from wcns_b200 import cases

pytestmark = pytest.mark.gpu


def test_get_interior_equals_ghosted_reads():
    from wcns_b200.solver import Wcns
    case = cases.small_channel_case()
    g = Wcns(case)
    g.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])
    g.step(2, history=False)
    names = ["r", "u", "v", "w", "p", "qke"]
    got = g.get_interior(names)
    for nb in range(1, case.nblocks + 1):
        for q, n in enumerate(names):
            np.testing.assert_array_equal(got[nb - 1][q], interior(g.get(n, nb), case.dims[nb - 1]))


def test_set_interior_writes_interior_only_and_skips_null_blocks():
    from wcns_b200.solver import Wcns
    case = cases.small_plate_case()
    g = Wcns(case)
    g.step(1, history=False)
    before = {(n, nb): g.get(n, nb).copy() for n in ("r", "p") for nb in range(1, case.nblocks + 1)}
    rng = np.random.default_rng(2)
    arrays = []
    for nb, (ni, nj, nk) in enumerate(case.dims, start=1):
        if nb == 3:
            arrays.append([None, None])  # block 3 keeps its values
        else:
            arrays.append([1.0 + 0.01 * rng.standard_normal((nk, nj, ni)), 0.7 + 0.01 * rng.standard_normal((nk, nj, ni))])
    g.set_interior(["r", "p"], arrays)
    for nb in range(1, case.nblocks + 1):
        d = case.dims[nb - 1]
        for q, n in enumerate(("r", "p")):
            after = g.get(n, nb)
            if nb == 3:
                np.testing.assert_array_equal(after, before[(n, nb)])
                continue
            np.testing.assert_array_equal(interior(after, d), arrays[nb - 1][q])
            mask = np.ones(after.shape, dtype=bool)
            mask[3:3 + d[2], 3:3 + d[1], 3:3 + d[0]] = False
            np.testing.assert_array_equal(after[mask], before[(n, nb)][mask])  # ghosts untouched
    # more fields than before: the staging buffer grows
    five = g.get_interior(["r", "u", "v", "w", "p"])
    for nb in range(1, case.nblocks + 1):
        np.testing.assert_array_equal(five[nb - 1][4], interior(g.get("p", nb), case.dims[nb - 1]))


def test_device_view_aliases_the_field():
    """wcns_field_device_ptr: a CUDA tensor over a block's field slice reads
    the field and writes into it (after the context's stream is idle)."""
    import torch
    from wcns_b200.solver import Wcns
    case = cases.small_plate_case()
    g = Wcns(case)
    g.step(1, history=False)
    g.sync()
    t = torch.as_tensor(g.device_view("p", 2), device="cuda")
    orig = g.get("p", 2)
    np.testing.assert_array_equal(t.cpu().numpy(), orig)
    before = g.get("r", 2)
    t.mul_(2.0)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(g.get("p", 2), 2.0 * orig)
    np.testing.assert_array_equal(g.get("r", 2), before)
