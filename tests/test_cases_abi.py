"""Host-side checks (no GPU): synthetic cases, the BC file format, the C ABI
surface of libwcns_b200.so and its argument validation."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from wcns_b200 import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "wcns_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wcns_[a-z0-9_]+)\s*\(", text)))


@pytest.mark.parametrize("make", [cases.plate_case, cases.small_plate_case, cases.vortex_case,
                                  cases.channel_case, cases.small_channel_case])
def test_bc_file_roundtrip(tmp_path, make):
    case = make()
    path = tmp_path / "bc.inp"
    cases.write_bc_file(str(path), case.dims, case.regions)
    dims, regions = cases.read_bc_file(str(path))
    assert [tuple(d) for d in dims] == [tuple(d) for d in case.dims]
    np.testing.assert_array_equal(regions, case.regions)


def test_channel_workload():
    """The 24-block SA channel: about 4 M points, every face of every block
    covered by exactly one region, walls on both channel walls."""
    case = cases.channel_case()
    assert case.nblocks == 24
    assert 3.8e6 < case.npoints < 4.3e6
    assert case.sa == {"timedt_turb": 10.0, "kmaxlim": 30000.0}
    for nb, (ni, nj, nk) in enumerate(case.dims, start=1):
        faces = {}
        for r in case.regions[case.regions[:, 0] == nb]:
            rng = [(abs(r[1 + 2 * d]), abs(r[2 + 2 * d])) for d in range(3)]
            d = [q for q in range(3) if rng[q][0] == rng[q][1] and (ni, nj, nk)[q] > 1][0]
            key = (d, rng[d][0])
            assert key not in faces
            assert all(sorted(rng[q]) == [1, (ni, nj, nk)[q]] for q in range(3) if q != d)
            faces[key] = int(r[7])
        assert len(faces) == 6
    assert sorted(set(case.regions[:, 7])) == [-1, 2, 3, 4]
    # the bump (height 0.05 H) lifts the lower wall at mid-length only: the
    # lower-wall blocks spanning x = length/2 reach its height, those whose
    # x range stays 1.5 H or more away from the middle stay flat
    lower = [nb for nb in range(1, 25) if any((case.regions[:, 0] == nb) & (case.regions[:, 7] == 2) & (case.regions[:, 3] == 1) & (case.regions[:, 4] == 1))]
    assert len(lower) == 12
    mid = 0.5 * float(max(case.xyz[nb - 1][0].max() for nb in lower))
    for nb in lower:
        x, y = case.xyz[nb - 1][0][:, 0, :], case.xyz[nb - 1][1][:, 0, :]
        if x.min() <= mid <= x.max():
            assert abs(float(y.max()) - 0.05) < 2e-3
        elif min(abs(float(x.min()) - mid), abs(float(x.max()) - mid)) >= 1.5:
            assert float(y.max()) < 1e-4


def test_plate_workload_size():
    case = cases.plate_case()
    assert case.nblocks == 8
    assert case.npoints == 228_888
    assert sorted(case.dims, reverse=True)[0] == (129, 65, 9)


def _face_points(xyz, rng):
    x, y, z = xyz
    sl = tuple(slice(abs(rng[d][0]) - 1, abs(rng[d][1])) for d in (2, 1, 0))  # arrays are (k, j, i)
    pts = np.stack([x[sl].ravel(), y[sl].ravel(), z[sl].ravel()], axis=1)
    return pts[np.lexsort(np.round(pts, 10).T[::-1])]


@pytest.mark.parametrize("make", [cases.plate_case, cases.small_plate_case, cases.small_channel_case])
def test_plate_interfaces_coincide(make):
    """Every one-to-one interface of the plate joins coincident points."""
    case = make()
    n = 0
    for r in case.regions:
        if r[7] >= 0:
            continue
        src = [(r[1], r[2]), (r[3], r[4]), (r[5], r[6])]
        dst = [(r[8], r[9]), (r[10], r[11]), (r[12], r[13])]
        a = _face_points(case.xyz[r[0] - 1], src)
        b = _face_points(case.xyz[r[14] - 1], dst)
        assert a.shape == b.shape
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-12)
        n += 1
    assert n > 0


def test_library_exports_every_header_function():
    from wcns_b200 import _lib
    names = header_functions()
    assert "wcns_create" in names and "wcns_step" in names and "wcns_residual_noalloc" in names
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_create_rejects_unsupported_scheme_before_device_work():
    from wcns_b200 import _lib
    from wcns_b200.solver import params_struct
    lib = _lib.load()
    case = cases.small_plate_case()
    case.params.nscheme = 45
    prm = params_struct(case.params)
    dims = (C.c_int * 3)(*case.dims[0])
    keep = [np.ascontiguousarray(a) for a in case.xyz[0]]
    xyz = (C.c_void_p * 3)(*[a.ctypes.data for a in keep])
    regs = np.ascontiguousarray(case.regions[case.regions[:, 0] == 1])
    h = C.c_void_p()
    rc = lib.wcns_create(C.byref(prm), 1, dims, xyz, 0, regs.ctypes.data_as(C.POINTER(C.c_int)), C.byref(h))
    assert rc == 5 and not h.value  # WCNS_ERR_UNSUPPORTED
    assert b"nscheme" in lib.wcns_last_error()


def test_noalloc_argument_checks_need_no_device():
    from wcns_b200 import _lib
    lib = _lib.load()
    assert lib.wcns_residual_noalloc(0, None, None, None, None, None, None) == 1
    nb = 300
    dims = (C.c_int * (3 * nb))(*([9] * (3 * nb)))
    ptrs = (C.c_void_p * (7 * nb))(*([8] * (7 * nb)))
    assert lib.wcns_residual_noalloc(nb, dims, ptrs, None, None, None, None) == 1
    assert b"maximum" in lib.wcns_last_error()
