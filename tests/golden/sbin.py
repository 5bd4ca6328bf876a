"""Reader for the ".sbin" array files written by oracle/ref_driver (test infrastructure).

Layout: a sequence of arrays, each [int32 name_len][name][int32 ndim][int64 dims...]
[float64 data] in little endian.
"""
import struct

import numpy as np


def read_sbin(path):
    out = {}
    with open(path, "rb") as f:
        b = f.read()
    o = 0
    while o < len(b):
        (nl,) = struct.unpack_from("<i", b, o)
        o += 4
        name = b[o:o + nl].decode()
        o += nl
        (nd,) = struct.unpack_from("<i", b, o)
        o += 4
        dims = struct.unpack_from("<%dq" % nd, b, o)
        o += 8 * nd
        n = int(np.prod(dims)) if nd else 1
        out[name] = np.frombuffer(b, dtype="<f8", count=n, offset=o).reshape(dims).copy()
        o += 8 * n
    return out
