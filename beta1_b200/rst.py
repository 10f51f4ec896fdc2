"""Reader/writer for the reference's MPCNSRST v1 restart layout.

Layout (src/5_io/IOModule_Bin.cpp:168-233 write, :234-387 read): 8-byte magic
"MPCNSRST", int32 version=1, int32 step, float64 time, int32 nblock,
int32 nfield, then per field: int32-length-prefixed name, int32 location,
int32 ncomp, int32 nghost, and per block: int32 lo[3], hi[3], int32 active,
then (if active) float64 values in (i, j, k, m) order, m fastest.

In memory a field is a dict {block: FieldArray}; ``FieldArray.data`` has shape
(ni, nj, nk, ncomp) over the half-open logical box [lo, hi), so logical index
(i, j, k) lives at data[i - lo[0], j - lo[1], k - lo[2]].
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field as dc_field
from typing import Dict, List, Optional

import numpy as np

MAGIC = b"MPCNSRST"

# Location codes as stored in the file (IOModule::LocToI32_, src/5_io/IOModule_Bin.cpp:62-85)
CELL, FACE_XI, FACE_ET, FACE_ZE, EDGE_XI, EDGE_ET, EDGE_ZE, NODE = range(8)


@dataclass
class FieldArray:
    lo: tuple
    hi: tuple
    data: Optional[np.ndarray]  # (ni, nj, nk, ncomp) float64, None if inactive

    def at(self, i, j, k, m=0):
        return self.data[i - self.lo[0], j - self.lo[1], k - self.lo[2], m]


@dataclass
class FieldRecord:
    name: str
    loc: int
    ncomp: int
    nghost: int
    blocks: List[FieldArray] = dc_field(default_factory=list)


@dataclass
class RestartFile:
    step: int
    time: float
    nblock: int
    fields: Dict[str, FieldRecord]


def read(path: str) -> RestartFile:
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != MAGIC:
        raise ValueError(f"{path}: not an MPCNSRST file")
    off = 8
    version, step = struct.unpack_from("<ii", buf, off)
    off += 8
    if version != 1:
        raise ValueError(f"{path}: unsupported version {version}")
    (time,) = struct.unpack_from("<d", buf, off)
    off += 8
    nblock, nfield = struct.unpack_from("<ii", buf, off)
    off += 8
    fields: Dict[str, FieldRecord] = {}
    for _ in range(nfield):
        (ln,) = struct.unpack_from("<i", buf, off)
        off += 4
        name = buf[off:off + ln].decode()
        off += ln
        loc, ncomp, nghost = struct.unpack_from("<iii", buf, off)
        off += 12
        rec = FieldRecord(name, loc, ncomp, nghost)
        for _b in range(nblock):
            vals = struct.unpack_from("<7i", buf, off)
            off += 28
            lo, hi, active = tuple(vals[0:3]), tuple(vals[3:6]), vals[6]
            if active:
                shape = (hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], ncomp)
                n = int(np.prod(shape))
                arr = np.frombuffer(buf, dtype="<f8", count=n, offset=off).reshape(shape).copy()
                off += 8 * n
            else:
                arr = None
            rec.blocks.append(FieldArray(lo, hi, arr))
        fields[name] = rec
    return RestartFile(step, time, nblock, fields)


def write(path: str, rf: RestartFile, names: Optional[List[str]] = None) -> None:
    names = list(rf.fields) if names is None else names
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<ii", 1, rf.step))
        f.write(struct.pack("<d", rf.time))
        f.write(struct.pack("<ii", rf.nblock, len(names)))
        for nm in names:
            rec = rf.fields[nm]
            b = nm.encode()
            f.write(struct.pack("<i", len(b)))
            f.write(b)
            f.write(struct.pack("<iii", rec.loc, rec.ncomp, rec.nghost))
            for fa in rec.blocks:
                f.write(struct.pack("<7i", *fa.lo, *fa.hi, 1 if fa.data is not None else 0))
                if fa.data is not None:
                    f.write(np.ascontiguousarray(fa.data, dtype="<f8").tobytes())


def extent(loc: int, ncell: tuple, nghost: int):
    """Logical [lo, hi) of a field at `loc` on a block of `ncell` cells
    (src/3_field/1_Field_Block.cpp:51-131)."""
    ni, nj, nk = ncell
    g = nghost
    plus = {
        CELL: (0, 0, 0), NODE: (1, 1, 1),
        FACE_XI: (1, 0, 0), FACE_ET: (0, 1, 0), FACE_ZE: (0, 0, 1),
        EDGE_XI: (0, 1, 1), EDGE_ET: (1, 0, 1), EDGE_ZE: (1, 1, 0),
    }[loc]
    lo = (-g, -g, -g)
    hi = (ni + plus[0] + g, nj + plus[1] + g, nk + plus[2] + g)
    return lo, hi
