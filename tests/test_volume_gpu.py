"""Filter outputs: NanoVDB grid topology and values, brick grid, volume
description — checked against the CPU oracle's payloads.

Active set (openvdb_backend.cpp:108-132): density > 0 or one of the 8 grid
corners, bit-exact.  Leaf values: the voxel payloads (inactive voxels hold the
background: zeros with ior 1).  The grid file is parsed here independently of
the library (documented NanoVDB 32.3 layout: 16-byte file header, 176-byte
metadata, name, GridData 672 B, TreeData 64 B, leaves of 16544 B).
"""
import ctypes as C
import json
import os
import struct

import numpy as np
import pytest

import oracle_lib as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from renderer2_b200 import _native as N  # noqa: E402
from renderer2_b200 import filter as F  # noqa: E402
from renderer2_b200 import scenes  # noqa: E402

N.lib.r2_filter_run_mesh.restype = C.c_int
N.lib.r2_filter_run_mesh.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_char_p,
                                     C.c_void_p]
N.lib.r2_nvdb_info.restype = C.c_int
N.lib.r2_nvdb_info.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
N.lib.r2_nvdb_lookup.restype = C.c_int
N.lib.r2_nvdb_lookup.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
N.lib.r2_brickgrid_info.restype = C.c_int
N.lib.r2_brickgrid_info.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]

BG = np.zeros(32, np.uint8)
BG[28:30] = np.frombuffer(np.float16(1.0).tobytes(), np.uint8)


def parse_nvdb_leaves(path):
    """Independent parse of the leaves of a NanoVDB Vec4d grid file."""
    raw = open(path, "rb").read()
    magic, version, grid_count, codec = struct.unpack_from("<QIHH", raw, 0)
    assert magic == 0x304244566f6e614e and grid_count == 1 and codec == 0
    grid_size = struct.unpack_from("<Q", raw, 16)[0]
    name_size = struct.unpack_from("<I", raw, 16 + 136)[0]
    g0 = 16 + 176 + name_size
    grid = raw[g0:g0 + grid_size]
    assert len(grid) == grid_size
    assert struct.unpack_from("<Q", grid, 0)[0] == 0x304244566f6e614e
    assert struct.unpack_from("<I", grid, 8 + 8 + 4 + 4 + 4 + 4 + 8 + 256 + 264 + 48 + 24 + 4)[0] == 18  # Vec4d
    node_off = struct.unpack_from("<4Q", grid, 672)
    node_cnt = struct.unpack_from("<3I", grid, 672 + 32)
    voxels = struct.unpack_from("<Q", grid, 672 + 56)[0]
    leaves = {}
    base = 672 + node_off[0]
    for i in range(node_cnt[0]):
        off = base + i * 16544
        bbmin = struct.unpack_from("<3i", grid, off)
        mask = np.frombuffer(grid, np.uint64, 8, off + 16)
        vals = np.frombuffer(grid, np.uint8, 512 * 32, off + 160).reshape(512, 32)
        origin = tuple(int(c) & ~7 for c in bbmin)
        leaves[origin] = (mask, vals)
    return leaves, voxels


def expected_leaves(comp, nv):
    nx, ny, nz = nv
    dens = comp[:, :4].copy().view(np.float32).reshape(-1)
    idx = np.arange(nx * ny * nz)
    x, y, z = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    corner = ((x == 0) | (x == nx - 1)) & ((y == 0) | (y == ny - 1)) & ((z == 0) | (z == nz - 1))
    active = (dens > 0) | corner
    return active, x, y, z


def run_lods(tmp_path, mesh, mat, prm, orient=(0, 1, 0), pos=(0, 0, 0), scale=(1, 1, 1), model="mesh"):
    pos3 = np.asarray(pos, np.float32)
    ori3 = np.asarray(orient, np.float32)
    sc3 = np.asarray(scale, np.float32)
    st = np.zeros(4)
    p = np.ascontiguousarray(mesh.positions, np.float32)
    ix = np.ascontiguousarray(mesh.indices, np.uint32)
    nr = np.ascontiguousarray(mesh.normals, np.float32)
    N.check(N.lib.r2_filter_run_mesh(N.ptr(p), mesh.nverts, N.ptr(ix), mesh.ntris, N.ptr(nr), C.byref(mat),
                                     N.ptr(pos3), N.ptr(ori3), N.ptr(sc3), C.byref(prm), str(tmp_path).encode(),
                                     model.encode(), N.ptr(st)))
    return st


def test_lod_outputs_topology_values_and_description(tmp_path):
    mesh = scenes.icosphere(4, 0.05, 1)
    mat = F.material()
    vs0 = scenes.voxel_size_for(mesh, 20)
    prm = F.params(samples_per_voxel=48, iterations=10, min_voxel_size=vs0, lods=3)
    st = run_lods(tmp_path, mesh, mat, prm)
    assert st[0] == 3
    desc = json.load(open(tmp_path / "volume_description.json"))
    assert list(desc.keys()) == ["mesh"]
    vs = np.float32(vs0)
    for lod in range(3):
        key = "%f" % float(vs)
        base = tmp_path / "mesh" / f"filtered_mesh_{key}"
        assert (tmp_path / "mesh" / f"filtered_mesh_{key}.nvdb").exists()
        assert (tmp_path / "mesh" / f"filtered_mesh_{key}.brickgrid").exists()
        # oracle payloads of this LOD
        lo = mesh.positions.min(0).astype(np.float32)
        hi = mesh.positions.max(0).astype(np.float32)
        g = O.setup_grid(lo, hi, N.identity43(), float(vs))
        nv = tuple(g.num_voxels[:])
        ow, oc = O.filter_voxels(mesh, O.material_from(mat), N.identity43(), g, O.params_from(prm), lod=lod)
        active, x, y, z = expected_leaves(oc, nv)
        leaves, nvox = parse_nvdb_leaves(str(base) + ".nvdb")
        assert nvox == int(active.sum())
        # every active voxel appears with its mask bit; every set bit is active
        seen = 0
        for (ox, oy, oz), (mask, vals) in leaves.items():
            for i in range(512):
                vx, vy, vz = ox + (i >> 6), oy + ((i >> 3) & 7), oz + (i & 7)
                bit = (int(mask[i >> 6]) >> (i & 63)) & 1
                inside = vx < nv[0] and vy < nv[1] and vz < nv[2]
                vid = vx + vy * nv[0] + vz * nv[0] * nv[1] if inside else -1
                exp = bool(active[vid]) if inside else False
                assert bit == exp
                if bit:
                    seen += 1
                    gv = vals[i].view(N.VOXEL_DTYPE)[0]
                    ov = oc[vid].view(N.VOXEL_DTYPE)[0]
                    for f in ["sigma", "r", "normal", "diffuse", "specular"]:
                        assert np.abs(gv[f].astype(int) - ov[f].astype(int)).max() <= 1
                    assert gv["ior"] == ov["ior"]
                else:
                    assert np.array_equal(vals[i], BG)
        assert seen == int(active.sum())
        # library reader agrees; index box spans the corners
        counts = np.zeros(4, np.uint64)
        ibb = np.zeros(6, np.int32)
        wbb = np.zeros(6, np.float64)
        m12 = np.zeros(12, np.float32)
        N.check(N.lib.r2_nvdb_info((str(base) + ".nvdb").encode(), N.ptr(counts), N.ptr(ibb), N.ptr(wbb), N.ptr(m12)))
        assert counts[3] == active.sum() and counts[0] == len(leaves)
        assert list(ibb) == [0, 0, 0, nv[0] - 1, nv[1] - 1, nv[2] - 1]
        assert np.array_equal(m12, np.array(g.index_to_model[:], np.float32))
        # volume description entry
        e = desc["mesh"][key]
        assert e["NumVoxels"] == list(nv)
        assert np.allclose(e["BBMin"], g.world_bb_min[:], atol=1e-6)
        assert np.allclose(e["P6"], e["BBMax"])
        # brick grid: bricks, ranges over the dilated 10^3 neighbourhood
        dims = np.zeros(7, np.uint32)
        mm = np.zeros(2, np.float32)
        N.check(N.lib.r2_brickgrid_info((str(base) + ".brickgrid").encode(), N.ptr(dims), N.ptr(mm), None, None, 0))
        nb = [int(-(-(-(-n // 8)) // 8) * 8) for n in nv]
        assert list(dims[:3]) == nb
        nB = nb[0] * nb[1] * nb[2]
        rng = np.zeros(nB, np.uint32)
        ind = np.zeros(nB, np.uint32)
        N.check(N.lib.r2_brickgrid_info((str(base) + ".brickgrid").encode(), None, None, N.ptr(ind), N.ptr(rng), nB))
        dens = np.where(active, oc[:, :4].copy().view(np.float32).reshape(-1), 0.0).reshape(nv[2], nv[1], nv[0])
        pad = np.zeros((nb[2] * 8 + 2, nb[1] * 8 + 2, nb[0] * 8 + 2), np.float32)
        pad[1:nv[2] + 1, 1:nv[1] + 1, 1:nv[0] + 1] = dens
        nonconst = 0
        for b in range(nB):
            bx, by, bz = b % nb[0], (b // nb[0]) % nb[1], b // (nb[0] * nb[1])
            blk = pad[bz * 8:bz * 8 + 10, by * 8:by * 8 + 10, bx * 8:bx * 8 + 10]
            lo16 = np.frombuffer(np.uint16(rng[b] & 0xFFFF).tobytes(), np.float16)[0]
            hi16 = np.frombuffer(np.uint16(rng[b] >> 16).tobytes(), np.float16)[0]
            assert abs(float(lo16) - float(np.float16(blk.min()))) <= 1e-3 * max(1.0, abs(float(blk.min())))
            assert abs(float(hi16) - float(np.float16(blk.max()))) <= 1e-3 * max(1.0, abs(float(blk.max())))
            if blk.max() != blk.min():
                nonconst += 1
            else:
                assert ind[b] == 0  # constant bricks keep no atlas slot
        assert nonconst == dims[6]
        vs = np.float32(vs * np.float32(2.0))


def test_nvdb_lookup_background_outside(tmp_path):
    mesh = scenes.icosphere(2, 0.05, 3)
    prm = F.params(samples_per_voxel=16, iterations=5, min_voxel_size=scenes.voxel_size_for(mesh, 8), lods=1)
    run_lods(tmp_path, mesh, F.material(), prm, model="small")
    path = [p for p in os.listdir(tmp_path / "small") if p.endswith(".nvdb")][0]
    coords = np.array([[-5, 0, 0], [100, 100, 100], [0, 0, 0]], np.int32)
    out = np.zeros(3, N.VOXEL_DTYPE)
    act = np.zeros(3, np.uint8)
    N.check(N.lib.r2_nvdb_lookup(str(tmp_path / "small" / path).encode(), N.ptr(coords), 3, N.ptr(out), N.ptr(act)))
    assert list(act) == [0, 0, 1]  # the origin is a grid corner, always active
    assert out[0].tobytes() == BG.tobytes() and out[1].tobytes() == BG.tobytes()


def test_corrupt_grid_file_rejected(tmp_path):
    p = tmp_path / "bad.nvdb"
    p.write_bytes(b"\x00" * 300)
    counts = np.zeros(4, np.uint64)
    st = N.lib.r2_nvdb_info(str(p).encode(), N.ptr(counts), None, None, None)
    assert N.lib.r2_status_string(st) == b"R2_ERR_IO"
    st = N.lib.r2_nvdb_info(str(tmp_path / "missing.nvdb").encode(), N.ptr(counts), None, None, None)
    assert N.lib.r2_status_string(st) == b"R2_ERR_IO"


def _density_grid_from_nvdb(path, nv):
    """Densities as the written grid stores them (inactive voxels: background 0), dens[z, y, x]."""
    leaves, _ = parse_nvdb_leaves(path)
    nx, ny, nz = nv
    dens = np.zeros((nz, ny, nx), np.float32)
    i = np.arange(512)
    dx, dy, dz = i >> 6, (i >> 3) & 7, i & 7
    for (ox, oy, oz), (mask, vals) in leaves.items():
        bits = (mask[i >> 6] >> (i & 63).astype(np.uint64)) & np.uint64(1)
        d = vals[:, :4].copy().view(np.float32).reshape(-1)
        x, y, z = ox + dx, oy + dy, oz + dz
        keep = (bits == 1) & (x < nx) & (y < ny) & (z < nz)
        dens[z[keep], y[keep], x[keep]] = d[keep]
    return dens


@pytest.mark.parametrize("n", [20, 37])
def test_brickgrid_archive_matches_reference_construction(tmp_path, n):
    """The .brickgrid written by the filter is the reference's cereal
    PortableBinary archive of CHostBrickGrid, parsed here independently, and
    every field equals the oracle's sequential restatement of the reference's
    construction (host_grid_brick.cpp:61-152) from the densities of the
    written NanoVDB grid: transform, n_bricks, min_maj, brick_counter,
    indirection, range, the atlas bytes and the three range mips, bit for bit.
    The library's own reader returns the same fields."""
    import brickgrid_io as BIO
    mesh = scenes.foliage(4000, 6, 0.7, 12)
    mat = F.material(diffuse=(0.2, 0.6, 0.1), specular=(0.04, 0.04, 0.04), alpha=0.4, ior=1.5)
    vs0 = scenes.voxel_size_for(mesh, n)
    prm = F.params(samples_per_voxel=32, iterations=8, min_voxel_size=vs0, lods=2)
    run_lods(tmp_path, mesh, mat, prm, model="leaves")
    vs = np.float32(vs0)
    for lod in range(2):
        base = tmp_path / "leaves" / f"filtered_mesh_{'%f' % float(vs)}"
        g = O.setup_grid(mesh.positions.min(0).astype(np.float32), mesh.positions.max(0).astype(np.float32),
                         N.identity43(), float(vs))
        nv = tuple(g.num_voxels[:])
        dens = _density_grid_from_nvdb(str(base) + ".nvdb", nv)
        ref = O.build_bricks(dens)
        got = BIO.parse(str(base) + ".brickgrid")
        assert np.array_equal(got["transform"], np.eye(4, dtype=np.float32).reshape(-1))
        assert np.array_equal(got["n_bricks"], ref["n_bricks"])
        assert np.array_equal(got["indirection_stride"], ref["n_bricks"])
        assert np.array_equal(got["min_maj"], ref["min_maj"])
        assert got["brick_counter"] == ref["brick_counter"] > 0
        assert np.array_equal(got["indirection"], ref["indirection"])
        assert np.array_equal(got["range"], ref["range"])
        assert np.array_equal(got["atlas_stride"], ref["atlas_stride"])
        assert np.array_equal(got["atlas"], ref["atlas"])
        assert len(got["mips"]) == 3
        for m, rm in zip(got["mips"], ref["mips"]):
            assert np.array_equal(m, rm)
        dims = np.zeros(7, np.uint32)
        mm = np.zeros(2, np.float32)
        N.check(N.lib.r2_brickgrid_info((str(base) + ".brickgrid").encode(), N.ptr(dims), N.ptr(mm), None, None, 0))
        assert list(dims) == list(ref["n_bricks"]) + list(ref["atlas_stride"]) + [ref["brick_counter"]]
        vs = np.float32(vs * np.float32(2.0))
