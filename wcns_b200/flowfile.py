"""Flow files: the reference's restart / output file of the primitive state.

write_flow_file_parallel and read_flow_file_parallel (parallel.f90:4073-4145,
3866-3992) write and read a Fortran unformatted sequential file, as gfortran
lays it out with the reference's `-fdefault-real-8`: every record is framed
by its length in bytes, a 4-byte little-endian integer before and after it.
  record 1            nout (integer*4), wholetime, roo, uoo, voo, woo, poo,
                      moo (real*8)
  record 1 + nb       block nb: r, u, v, w, p, T interleaved per point, i
                      fastest, then j, then k (real*8)
The reader skips the free-stream values, as the reference does, and takes
nout and wholetime.  A record longer than 2^31 - 1 bytes (gfortran would
split it into subrecords) is refused.

`write_flow(path, g)` reads the interior state of every block from a GPU
context with one synchronisation (wcns_get_flow); `load_flow(g, path)` puts
a file's state into a context's interior points (wcns_set_interior), whose
ghosts the next step's boundary conditions fill, as init_nstart1 leaves them.
"""
from __future__ import annotations

import struct

import numpy as np

_MAX = 2 ** 31 - 1


def _write_record(f, payload: bytes):
    if len(payload) > _MAX:
        raise ValueError(f"a record of {len(payload)} bytes needs subrecords, which this writer does not produce")
    n = struct.pack("<i", len(payload))
    f.write(n)
    f.write(payload)
    f.write(n)


def _read_record(f) -> bytes:
    head = f.read(4)
    if len(head) != 4:
        raise EOFError("end of file before a record")
    (n,) = struct.unpack("<i", head)
    if n < 0:
        raise ValueError("a subrecord marker: records over 2 GiB are not supported")
    payload = f.read(n)
    tail = f.read(4)
    if len(payload) != n or tail != head:
        raise ValueError("record markers do not match: not a flow file of this layout")
    return payload


def write_flow_arrays(path, blocks, nout, wholetime, freestream, moo):
    """blocks[nb-1] = six arrays (nk, nj, ni): r, u, v, w, p, T;
    freestream = (roo, uoo, voo, woo, poo)."""
    with open(path, "wb") as f:
        _write_record(f, struct.pack("<i7d", int(nout), float(wholetime), *[float(v) for v in freestream], float(moo)))
        for arrs in blocks:
            if len(arrs) != 6:
                raise ValueError("six arrays per block: r, u, v, w, p, T")
            inter = np.stack([np.asarray(a, dtype="<f8") for a in arrs], axis=-1)  # (nk, nj, ni, 6)
            _write_record(f, np.ascontiguousarray(inter).tobytes())


def read_flow(path, dims):
    """({"nout", "wholetime", "freestream", "moo"}, [six arrays (nk, nj, ni)
    per block]) of a flow file of blocks with dimensions dims."""
    with open(path, "rb") as f:
        head = _read_record(f)
        if len(head) != 4 + 7 * 8:
            raise ValueError("the first record is not nout, wholetime and six free-stream values")
        v = struct.unpack("<i7d", head)
        header = {"nout": v[0], "wholetime": v[1], "freestream": tuple(v[2:7]), "moo": v[7]}
        blocks = []
        for ni, nj, nk in dims:
            rec = _read_record(f)
            if len(rec) != 6 * 8 * ni * nj * nk:
                raise ValueError(f"a block record of {len(rec)} bytes does not match {ni} x {nj} x {nk} points")
            a = np.frombuffer(rec, dtype="<f8").reshape(nk, nj, ni, 6)
            blocks.append([np.ascontiguousarray(a[..., m]) for m in range(6)])
    return header, blocks


def write_flow(path, g, nout=0, wholetime=0.0):
    """The context's interior state as a flow file (write_flow_file_parallel)."""
    p = g.case.params
    write_flow_arrays(path, g.get_flow(), nout, wholetime, p.freestream(), p.moo)


def load_flow(g, path):
    """A flow file's state into the context's interior points
    (read_flow_file_parallel); returns the header."""
    header, blocks = read_flow(path, g.dims)
    g.set_interior(["r", "u", "v", "w", "p", "t"], blocks)
    return header
