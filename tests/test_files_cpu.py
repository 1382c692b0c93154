"""File readers reject corrupt or missing inputs with status codes (no GPU needed)."""
import ctypes as C

import numpy as np

from renderer2_b200 import _native as N

N.lib.r2_nvdb_info.restype = C.c_int
N.lib.r2_nvdb_info.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
N.lib.r2_brickgrid_info.restype = C.c_int
N.lib.r2_brickgrid_info.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]


def test_corrupt_and_missing_nvdb(tmp_path):
    counts = np.zeros(4, np.uint64)
    p = tmp_path / "bad.nvdb"
    p.write_bytes(b"\x00" * 300)
    assert N.lib.r2_status_string(N.lib.r2_nvdb_info(str(p).encode(), N.ptr(counts), None, None, None)) == b"R2_ERR_IO"
    st = N.lib.r2_nvdb_info(str(tmp_path / "missing.nvdb").encode(), N.ptr(counts), None, None, None)
    assert N.lib.r2_status_string(st) == b"R2_ERR_IO"
    # a valid header with a truncated grid body
    hdr = (0x304244566f6e614e).to_bytes(8, "little") + ((32 << 21) | (3 << 10) | 3).to_bytes(4, "little")
    hdr += (1).to_bytes(2, "little") + (0).to_bytes(2, "little")
    meta = bytearray(176)
    meta[0:8] = (100000).to_bytes(8, "little")
    meta[136:140] = (1).to_bytes(4, "little")
    p.write_bytes(hdr + bytes(meta) + b"\x00" + b"\x01" * 64)
    assert N.lib.r2_status_string(N.lib.r2_nvdb_info(str(p).encode(), N.ptr(counts), None, None, None)) == b"R2_ERR_IO"


def test_corrupt_brickgrid(tmp_path):
    p = tmp_path / "bad.brickgrid"
    p.write_bytes(b"R2BRICK1" + b"\xff" * 40)
    dims = np.zeros(7, np.uint32)
    st = N.lib.r2_brickgrid_info(str(p).encode(), N.ptr(dims), None, None, None, 0)
    assert N.lib.r2_status_string(st) == b"R2_ERR_IO"
