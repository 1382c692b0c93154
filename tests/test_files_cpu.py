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


def test_library_reads_a_reference_layout_brickgrid(tmp_path):
    """A .brickgrid archive written here in the reference's cereal layout, from
    the oracle's construction of a sparse random density grid, is read by the
    library's reader with every field intact."""
    import brickgrid_io as BIO
    import oracle_lib as O
    from renderer2_b200 import _native as N
    rng = np.random.default_rng(3)
    dens = np.where(rng.uniform(size=(37, 21, 50)) < 0.2, rng.lognormal(0, 1, (37, 21, 50)), 0.0).astype(np.float32)
    g = O.build_bricks(dens)
    assert g["brick_counter"] > 0
    p = tmp_path / "grid.brickgrid"
    BIO.write(p, g)
    back = BIO.parse(p)
    assert np.array_equal(back["atlas"], g["atlas"]) and back["brick_counter"] == g["brick_counter"]
    N.lib.r2_brickgrid_info.argtypes = [C.c_char_p] + [C.c_void_p] * 4 + [C.c_size_t]
    dims = np.zeros(7, np.uint32)
    mm = np.zeros(2, np.float32)
    nB = int(np.prod(g["n_bricks"].astype(np.int64)))
    ind = np.zeros(nB, np.uint32)
    rg = np.zeros(nB, np.uint32)
    N.check(N.lib.r2_brickgrid_info(str(p).encode(), N.ptr(dims), N.ptr(mm), N.ptr(ind), N.ptr(rg), nB))
    assert list(dims[:3]) == list(g["n_bricks"]) and list(dims[3:6]) == list(g["atlas_stride"])
    assert dims[6] == g["brick_counter"]
    assert np.array_equal(mm, g["min_maj"])
    assert np.array_equal(ind, g["indirection"]) and np.array_equal(rg, g["range"])
    # a truncated archive is refused
    (tmp_path / "cut.brickgrid").write_bytes(p.read_bytes()[:-3])
    st = N.lib.r2_brickgrid_info(str(tmp_path / "cut.brickgrid").encode(), N.ptr(dims), None, None, None, 0)
    assert N.lib.r2_status_string(st) == b"R2_ERR_IO"
