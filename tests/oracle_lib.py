"""ctypes view of the CPU oracle (oracle/_build/liboracle.so) — the checker.

Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline legs use it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "_build", "liboracle.so")


def ensure_built() -> str:
    if not os.path.exists(ORACLE_LIB) or any(
            os.path.getmtime(os.path.join(ORACLE_DIR, f)) > os.path.getmtime(ORACLE_LIB)
            for f in os.listdir(ORACLE_DIR) if f.endswith((".c", ".h"))):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    return ORACLE_LIB


class Grid(C.Structure):
    _fields_ = [("num_voxels", C.c_int32 * 3), ("index_to_model", C.c_float * 12),
                ("model_to_index", C.c_float * 12), ("model_to_world", C.c_float * 12),
                ("world_to_model", C.c_float * 12), ("world_bb_min", C.c_float * 3),
                ("world_bb_max", C.c_float * 3), ("voxel_size", C.c_float)]


class Material(C.Structure):
    _fields_ = [("diffuse", C.c_float * 3), ("specular", C.c_float * 3), ("alpha_x", C.c_float),
                ("alpha_y", C.c_float), ("eta_i", C.c_float), ("eta_t", C.c_float),
                ("diffuse_roughness", C.c_float), ("pad", C.c_float)]


class Params(C.Structure):
    _fields_ = [("min_voxel_size", C.c_float), ("lods", C.c_uint32), ("samples_per_voxel", C.c_uint32),
                ("sigma_t", C.c_float), ("estimation_iterations", C.c_uint32), ("alpha", C.c_float),
                ("clip_rays", C.c_uint32), ("seed", C.c_uint32), ("sggx_projection", C.c_uint32),
                ("sggx_floor", C.c_float)]


def _load():
    lib = C.CDLL(ensure_built())
    P = C.c_void_p
    lib.orc_philox4x32_10.argtypes = [P, P, P]
    lib.orc_sincos_turns.argtypes = [C.c_float, P, P]
    lib.orc_build_bvh.argtypes = [P, C.c_uint32, P, C.c_uint32, P, P, P]
    lib.orc_build_bvh.restype = C.c_int
    lib.orc_trace.argtypes = [P, P] + [C.c_float] * 7 + [P, P, P]
    lib.orc_trace.restype = C.c_int
    lib.orc_setup_grid.argtypes = [P, P, P, C.c_float, P]
    lib.orc_filter.argtypes = [P, C.c_uint32, P, C.c_uint32, P, P, P, P, P, C.c_uint32, C.c_uint64, C.c_uint64, P,
                               P, C.c_int]
    lib.orc_filter.restype = C.c_int
    lib.orc_filter_tex.argtypes = [P, C.c_uint32, P, C.c_uint32, P, P, P, P, P, P, P, P, P, P, C.c_uint32, C.c_uint64,
                                   C.c_uint64, P, P, C.c_int]
    lib.orc_filter_tex.restype = C.c_int
    lib.orc_encode.argtypes = [P, P]
    return lib


lib = _load()


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib.orc_philox4x32_10(_p(c), _p(k), _p(out))
    return out


def sincos_turns(u):
    s = C.c_float()
    c = C.c_float()
    lib.orc_sincos_turns(C.c_float(u), C.byref(s), C.byref(c))
    return s.value, c.value


def build_bvh(world_pos, idx):
    pos = np.ascontiguousarray(world_pos, np.float32)
    ix = np.ascontiguousarray(idx, np.uint32)
    n = ix.shape[0]
    nodes = np.zeros((max(n - 1, 1), 16), np.int32)
    order = np.zeros(n, np.uint32)
    tris = np.zeros((n, 12), np.float32)
    h = lib.orc_build_bvh(_p(pos), pos.shape[0], _p(ix), n, _p(nodes), _p(order), _p(tris))
    return nodes, order, tris, h


def trace(nodes, tris, o, d, tmax):
    t = C.c_float()
    b1 = C.c_float()
    b2 = C.c_float()
    tri = lib.orc_trace(_p(nodes), _p(tris), *[float(x) for x in o], *[float(x) for x in d], float(tmax),
                        C.byref(t), C.byref(b1), C.byref(b2))
    return tri, t.value, b1.value, b2.value


def setup_grid(lo, hi, m2w, vs):
    g = Grid()
    lo = np.ascontiguousarray(lo, np.float32)
    hi = np.ascontiguousarray(hi, np.float32)
    m = np.ascontiguousarray(m2w, np.float32)
    lib.orc_setup_grid(_p(lo), _p(hi), _p(m), C.c_float(vs), C.byref(g))
    return g


def material_from(native_mat) -> Material:
    m = Material()
    C.memmove(C.byref(m), C.byref(native_mat), C.sizeof(Material))
    return m


def params_from(native_params) -> Params:
    p = Params()
    C.memmove(C.byref(p), C.byref(native_params), C.sizeof(Params))
    return p


def grid_from(native_grid) -> Grid:
    g = Grid()
    C.memmove(C.byref(g), C.byref(native_grid), C.sizeof(Grid))
    return g


def filter_voxels(mesh, mat, m2w, grid, prm, v0=0, v1=None, lod=0, threads=0, tex=None):
    """Oracle filter of voxels [v0, v1): (wide float64 (n, 20), compact uint8 (n, 32)).
    tex (nullable): dict(uv=(n, 2), albedo / specular / normal / alpha = PNG path)."""
    nvox = int(np.prod(np.array(grid.num_voxels[:], np.int64)))
    v1 = nvox if v1 is None else v1
    pos = np.ascontiguousarray(mesh.positions, np.float32)
    idx = np.ascontiguousarray(mesh.indices, np.uint32)
    nrm = np.ascontiguousarray(mesh.normals, np.float32)
    m2w = np.ascontiguousarray(m2w, np.float32)
    wide = np.zeros((v1 - v0, 20), np.float64)
    comp = np.zeros((v1 - v0, 32), np.uint8)
    keep, maps, uv = [], [None] * 4, None
    if tex is not None:
        from renderer2_b200 import pipeline as P
        uv = np.ascontiguousarray(tex["uv"], np.float32)
        for k, key in enumerate(("albedo", "specular", "normal", "alpha")):
            if tex.get(key):
                rgba, ch = P.read_png(tex[key])
                ot = OTexture(rgba.shape[1], rgba.shape[0], ch, rgba.ctypes.data)
                keep += [rgba, ot]
                maps[k] = C.byref(ot)
    r = lib.orc_filter_tex(_p(pos), pos.shape[0], _p(idx), idx.shape[0], _p(nrm), _p(uv), C.byref(mat), *maps,
                           _p(m2w), C.byref(grid), C.byref(prm), lod, v0, v1, _p(wide), _p(comp), threads)
    assert r >= 0, f"oracle filter failed ({r})"
    return wide, comp


# ---------------------------------------------------------------- path tracer oracle

class OTexture(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("channels", C.c_int), ("rgba", C.c_void_p)]


class OMesh(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("nverts", C.c_uint32), ("indices", C.c_void_p), ("ntris", C.c_uint32),
                ("normals", C.c_void_p), ("model_to_world", C.c_float * 12), ("material", Material),
                ("uvs", C.c_void_p), ("albedo", C.c_void_p), ("specular", C.c_void_p), ("normal", C.c_void_p),
                ("alpha", C.c_void_p), ("asset", C.c_uint32)]


class OShape(C.Structure):
    _fields_ = [("type", C.c_int), ("center", C.c_float * 3), ("radius", C.c_float), ("normal", C.c_float * 3),
                ("material", Material)]


class OCamera(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("fov_deg", C.c_float), ("pos", C.c_float * 3),
                ("look_at", C.c_float * 3), ("up", C.c_float * 3)]


class OMedium(C.Structure):
    _fields_ = [("path", C.c_char_p), ("sigma_a", C.c_float * 3), ("sigma_s", C.c_float * 3), ("pos", C.c_float * 3),
                ("orientation", C.c_float * 3), ("scaling", C.c_float * 3), ("hg", C.c_int), ("g", C.c_float)]


lib.orc_render.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                           C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_int,
                           C.c_void_p, C.c_uint32, C.c_uint32]
lib.orc_render.restype = C.c_int
lib.orc_t_log.argtypes = [C.c_float]
lib.orc_t_log.restype = C.c_float
lib.orc_env_sample.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
lib.orc_env_le.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]


def render(scene_desc, cam, spp, max_depth, seed, p0=0, p1=None, threads=0, want_var=False, flags=0,
           instancing=True):
    """scene_desc: dict(meshes=[(Mesh, native material, m2w)], shapes=[(kind, center, radius, normal, material)],
    media=[(path, sigma_a, sigma_s, pos, orientation, scaling)], env=(H, W, 3) float32).
    With instancing, meshes sharing their mesh and material objects are instances of one asset, as the
    library's scene builder makes them.  Returns rgb (n, 3) [, var (n, 3)] for pixels [p0, p1)."""
    keep = []
    asset_of = {}
    if instancing:
        from renderer2_b200 import render_scenes as RS
        for a, group in enumerate(RS.mesh_groups(scene_desc)):
            for k in group:
                asset_of[k] = a + 1
    media = (OMedium * max(1, len(scene_desc.get("media", []))))()
    for i, med in enumerate(scene_desc.get("media", [])):
        path, sa, ss, pos, ori, sc = med[:6]
        if len(med) > 6 and med[6] is not None:  # Henyey-Greenstein asymmetry g
            media[i].hg = 1
            media[i].g = float(med[6])
        pb = str(path).encode()
        keep.append(pb)
        media[i].path = pb
        media[i].sigma_a[:] = list(map(float, sa))
        media[i].sigma_s[:] = list(map(float, ss))
        media[i].pos[:] = list(map(float, pos))
        media[i].orientation[:] = list(map(float, ori))
        media[i].scaling[:] = list(map(float, sc))
    meshes = (OMesh * max(1, len(scene_desc.get("meshes", []))))()
    for i, entry in enumerate(scene_desc.get("meshes", [])):
        mesh, mat, m2w = entry[:3]
        tex = entry[3] if len(entry) > 3 else None
        if tex is not None:  # texture coordinates and texture maps decoded by the library's PNG reader
            from renderer2_b200 import pipeline as P
            uv = np.ascontiguousarray(tex["uv"], np.float32)
            keep.append(uv)
            meshes[i].uvs = uv.ctypes.data
            for key in ("albedo", "specular", "normal", "alpha"):
                if tex.get(key):
                    rgba, ch = P.read_png(tex[key])
                    ot = OTexture(rgba.shape[1], rgba.shape[0], ch, rgba.ctypes.data)
                    keep += [rgba, ot]
                    setattr(meshes[i], key, C.addressof(ot))
        pos = np.ascontiguousarray(mesh.positions, np.float32)
        idx = np.ascontiguousarray(mesh.indices, np.uint32)
        nrm = np.ascontiguousarray(mesh.normals, np.float32)
        keep += [pos, idx, nrm]
        meshes[i].positions = pos.ctypes.data
        meshes[i].nverts = pos.shape[0]
        meshes[i].indices = idx.ctypes.data
        meshes[i].ntris = idx.shape[0]
        meshes[i].normals = nrm.ctypes.data
        meshes[i].model_to_world[:] = [float(x) for x in np.asarray(m2w, np.float32)]
        meshes[i].material = material_from(mat)
        meshes[i].asset = asset_of.get(i, 0)
    shapes = (OShape * max(1, len(scene_desc.get("shapes", []))))()
    for i, (kind, c, r, n, mat) in enumerate(scene_desc.get("shapes", [])):
        shapes[i].type = kind
        shapes[i].center[:] = list(map(float, c))
        shapes[i].radius = float(r)
        shapes[i].normal[:] = list(map(float, n))
        shapes[i].material = material_from(mat)
    env = np.ascontiguousarray(scene_desc["env"], np.float32)
    oc = OCamera()
    C.memmove(C.byref(oc), C.byref(cam), C.sizeof(OCamera))
    npix = cam.width * cam.height
    p1 = npix if p1 is None else p1
    rgb = np.zeros((p1 - p0, 3), np.float32)
    var = np.zeros((p1 - p0, 3), np.float64) if want_var else None
    r = lib.orc_render(C.addressof(meshes), len(scene_desc.get("meshes", [])), C.addressof(shapes),
                       len(scene_desc.get("shapes", [])), env.ctypes.data, env.shape[1], env.shape[0], C.byref(oc),
                       spp, max_depth, seed, p0, p1, rgb.ctypes.data, _p(var), threads, C.addressof(media),
                       len(scene_desc.get("media", [])), flags)
    assert r == 0, f"oracle render failed ({r})"
    return (rgb, var) if want_var else rgb


lib.orc_tonemap.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p]
lib.orc_tonemap.restype = None


def tonemap(linear, gamma):
    """Oracle output stage: (tonemapped floats, bytes) of an (H, W, 3) frame."""
    lin = np.ascontiguousarray(linear, np.float32)
    out = np.zeros_like(lin)
    by = np.zeros(lin.shape, np.uint8)
    lib.orc_tonemap(lin.ctypes.data, lin.shape[1], lin.shape[0], float(gamma), out.ctypes.data, by.ctypes.data)
    return out, by


lib.orc_select_lods.restype = C.c_int
lib.orc_select_lods.argtypes = [C.c_void_p] * 4 + [C.c_uint32] + [C.c_void_p] * 3 + [C.c_uint32, C.c_double,
                                                                                      C.c_double, C.c_void_p,
                                                                                      C.c_void_p]


def select_lods(cam_rec, lods, first, count, tree_pos, tree_scaling, tree_model, min_lod, covered_pixels,
                want_diag=False):
    """selectLOD per tree (orc_select_lods): LOD index or -1; with want_diag
    also (covered pixels, hull area, 0) per tree."""
    pos = np.ascontiguousarray(np.asarray(tree_pos, np.float64).reshape(-1, 3))
    sc = np.ascontiguousarray(np.asarray(tree_scaling, np.float64).reshape(-1))
    mdl = np.ascontiguousarray(np.asarray(tree_model, np.uint32).reshape(-1))
    first = np.ascontiguousarray(first, np.uint32)
    count = np.ascontiguousarray(count, np.uint32)
    out = np.zeros(len(sc), np.int32)
    diag = np.zeros((len(sc), 3)) if want_diag else None
    rc = lib.orc_select_lods(_p(cam_rec), _p(lods), _p(first), _p(count), len(first), _p(pos), _p(sc), _p(mdl),
                             len(sc), float(min_lod), float(covered_pixels), _p(out), _p(diag))
    assert rc == 0
    return (out, diag) if want_diag else out


def build_bricks(dens):
    """The reference's brick grid (CHostBrickGrid) of a density grid dens[z, y, x] (float32), built by the oracle
    one brick after the other: dict of the archive's fields."""
    d = np.ascontiguousarray(dens, np.float32)
    nz, ny, nx = d.shape
    nb = np.zeros(3, np.uint32)
    P = C.c_void_p
    lib.orc_build_bricks.argtypes = [P, C.c_int, C.c_int, C.c_int] + [P] * 10
    lib.orc_build_bricks.restype = C.c_int
    assert lib.orc_build_bricks(_p(d), nx, ny, nz, _p(nb), *([None] * 9)) == 0
    nB = int(nb[0]) * int(nb[1]) * int(nb[2])
    ind = np.zeros(nB, np.uint32)
    rng = np.zeros(nB, np.uint32)
    mips = [np.zeros(int(nb[0] >> (i + 1)) * int(nb[1] >> (i + 1)) * int(nb[2] >> (i + 1)), np.uint32)
            for i in range(3)]
    atlas = np.zeros(nB * 512, np.uint8)
    ad = np.zeros(3, np.uint32)
    cnt = np.zeros(1, np.uint64)
    mm = np.zeros(2, np.float32)
    assert lib.orc_build_bricks(_p(d), nx, ny, nz, _p(nb), _p(ind), _p(rng), _p(mips[0]), _p(mips[1]), _p(mips[2]),
                                _p(atlas), _p(ad), _p(cnt), _p(mm)) == 0
    return {"n_bricks": nb, "min_maj": mm, "brick_counter": int(cnt[0]), "indirection": ind, "range": rng,
            "atlas_stride": ad, "atlas": atlas[:int(ad[0]) * int(ad[1]) * int(ad[2])], "mips": mips}
