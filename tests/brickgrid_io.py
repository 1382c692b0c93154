"""The reference's .brickgrid file, read and written here independently of the
library: a cereal 1.3.2 PortableBinary archive of CHostBrickGrid
(raytracer/src/grid_brick/serialization.cpp:37-40, Buf3D at :32-34).

cereal's PortableBinaryOutputArchive first writes one byte telling whether
the data is little-endian, then every arithmetic value in that order of bytes;
a std::vector of arithmetic type is a uint64 element count followed by the
elements, a std::vector of class type a uint64 count followed by each
element's fields; std::pair and std::atomic<size_t> serialise their values;
glm vectors and matrices are serialised component by component (mat4 as its
four columns).
"""
from __future__ import annotations

import struct

import numpy as np


def parse(path) -> dict:
    raw = open(path, "rb").read()
    off = 0

    def take(fmt):
        nonlocal off
        v = struct.unpack_from("<" + fmt, raw, off)
        off += struct.calcsize("<" + fmt)
        return v

    def buf3d(dtype):
        nonlocal off
        stride = np.array(take("3I"), np.uint32)
        (n,) = take("Q")
        assert n == int(np.prod(stride.astype(np.int64)))
        a = np.frombuffer(raw, dtype, n, off).copy()
        off += n * np.dtype(dtype).itemsize
        return stride, a

    (little,) = take("B")
    assert little == 1
    g = {"transform": np.array(take("16f"), np.float32), "n_bricks": np.array(take("3I"), np.uint32),
         "min_maj": np.array(take("2f"), np.float32), "brick_counter": take("Q")[0]}
    g["indirection_stride"], g["indirection"] = buf3d(np.uint32)
    g["range_stride"], g["range"] = buf3d(np.uint32)
    g["atlas_stride"], g["atlas"] = buf3d(np.uint8)
    (nm,) = take("Q")
    g["mips"] = []
    g["mip_strides"] = []
    for _ in range(nm):
        s, a = buf3d(np.uint32)
        g["mip_strides"].append(s)
        g["mips"].append(a)
    assert off == len(raw), "trailing bytes"
    return g


def write(path, g: dict) -> None:
    """Archive of the fields of the oracle's construction (oracle_lib.build_bricks)."""
    nb = np.asarray(g["n_bricks"], np.uint32)
    out = [struct.pack("<B", 1), np.eye(4, dtype=np.float32).tobytes(order="F"), nb.tobytes(),
           np.asarray(g["min_maj"], np.float32).tobytes(), struct.pack("<Q", int(g["brick_counter"]))]

    def buf3d(stride, a):
        out.append(np.asarray(stride, np.uint32).tobytes())
        out.append(struct.pack("<Q", a.size))
        out.append(np.ascontiguousarray(a).tobytes())

    buf3d(nb, np.asarray(g["indirection"], np.uint32))
    buf3d(nb, np.asarray(g["range"], np.uint32))
    buf3d(g["atlas_stride"], np.asarray(g["atlas"], np.uint8))
    out.append(struct.pack("<Q", len(g["mips"])))
    for i, m in enumerate(g["mips"]):
        buf3d(nb >> (i + 1), np.asarray(m, np.uint32))
    with open(path, "wb") as fh:
        fh.write(b"".join(out))
