"""Flow files (wcns_b200/flowfile.py): the reference's unformatted restart
file of the primitive state (write_flow_file_parallel / read_flow_file_parallel,
parallel.f90:4073-4145, 3866-3992).

CPU: the byte layout of a small file built by hand (record markers, the
header record, r..T interleaved per point with i fastest), the round trip,
and the refusals (wrong block size, damaged markers).
GPU: a context's state written and loaded into a fresh context, which then
steps exactly as the original does (a restart)."""
import struct

import numpy as np
import pytest

from wcns_b200 import cases, flowfile


def test_byte_layout_by_hand(tmp_path):
    ni, nj, nk = 2, 3, 1
    arrs = [np.arange(nk * nj * ni, dtype=float).reshape(nk, nj, ni) + 10 * m for m in range(6)]
    p = tmp_path / "flow.dat"
    flowfile.write_flow_arrays(p, [arrs], 7, 1.5, (1.0, 0.9, 0.1, 0.0, 2.5), 0.6)
    raw = p.read_bytes()
    head = struct.pack("<i7d", 7, 1.5, 1.0, 0.9, 0.1, 0.0, 2.5, 0.6)
    body = b"".join(struct.pack("<6d", *[arrs[m][k, j, i] for m in range(6)])
                    for k in range(nk) for j in range(nj) for i in range(ni))
    want = (struct.pack("<i", len(head)) + head + struct.pack("<i", len(head)) +
            struct.pack("<i", len(body)) + body + struct.pack("<i", len(body)))
    assert raw == want


def test_round_trip_and_refusals(tmp_path):
    dims = [(4, 3, 2), (5, 2, 3)]
    rng = np.random.default_rng(0)
    blocks = [[rng.standard_normal((nk, nj, ni)) for _ in range(6)] for ni, nj, nk in dims]
    p = tmp_path / "flow.dat"
    flowfile.write_flow_arrays(p, blocks, 12, 3.25, (1.0, 1.0, 0.0, 0.0, 1.98), 0.6)
    header, got = flowfile.read_flow(p, dims)
    assert header["nout"] == 12 and header["wholetime"] == 3.25 and header["moo"] == 0.6
    for a, b in zip(blocks, got):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
    with pytest.raises(ValueError):
        flowfile.read_flow(p, [(4, 3, 2), (5, 2, 4)])
    raw = bytearray(p.read_bytes())
    raw[-1] ^= 0xFF
    bad = tmp_path / "bad.dat"
    bad.write_bytes(bytes(raw))
    with pytest.raises(ValueError):
        flowfile.read_flow(bad, dims)


@pytest.mark.gpu
def test_restart_from_flow_file_steps_like_the_original(tmp_path):
    from wcns_b200.solver import Wcns
    case = cases.small_plate_case()
    a = Wcns(case)
    a.step(3, history=False)
    p = tmp_path / "flow.dat"
    flowfile.write_flow(p, a, nout=3)
    b = Wcns(case)
    header = flowfile.load_flow(b, p)
    assert header["nout"] == 3
    ha, hb = a.step(2), b.step(2)
    np.testing.assert_array_equal(ha, hb)
    for nb in range(1, case.nblocks + 1):
        for f in ("r", "u", "v", "w", "p"):
            np.testing.assert_array_equal(a.get(f, nb)[3:-3, 3:-3, 3:-3], b.get(f, nb)[3:-3, 3:-3, 3:-3])
