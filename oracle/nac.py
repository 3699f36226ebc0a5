"""Reader/writer for the "named array" container (.nac) used by the oracle probes.

Test infrastructure only.  Layout, repeated until EOF:
    int32 name_len; bytes name; char dtype ('i' = int32, 'd' = float64);
    int32 ndim; int32 shape[ndim]; raw little-endian data.
The C++ side lives in oracle/probe/probe_common.h.
"""
from __future__ import annotations

import struct

import numpy as np


def read_nac(path: str) -> dict[str, np.ndarray]:
    out: dict[str, np.ndarray] = {}
    with open(path, "rb") as f:
        buf = f.read()
    pos = 0
    while pos < len(buf):
        (n,) = struct.unpack_from("<i", buf, pos)
        pos += 4
        name = buf[pos:pos + n].decode()
        pos += n
        dt = chr(buf[pos])
        pos += 1
        (nd,) = struct.unpack_from("<i", buf, pos)
        pos += 4
        shape = struct.unpack_from("<%di" % nd, buf, pos)
        pos += 4 * nd
        count = int(np.prod(shape)) if nd else 1
        dtype = np.int32 if dt == "i" else np.float64
        arr = np.frombuffer(buf, dtype=dtype, count=count, offset=pos).reshape(shape).copy()
        pos += arr.nbytes
        out[name] = arr
    return out


def write_nac(path: str, arrays: dict[str, np.ndarray]) -> None:
    with open(path, "wb") as f:
        for name, a in arrays.items():
            a = np.asarray(a)
            if a.dtype.kind in "iub":
                a = a.astype(np.int32)
                dt = b"i"
            else:
                a = a.astype(np.float64)
                dt = b"d"
            nb = name.encode()
            f.write(struct.pack("<i", len(nb)) + nb + dt)
            f.write(struct.pack("<i", a.ndim) + struct.pack("<%di" % a.ndim, *a.shape))
            f.write(np.ascontiguousarray(a).tobytes())
