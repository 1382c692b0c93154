"""Generates tests/golden/ref_math.json from the reference's own headers.

Builds oracle/_ref/libr2ref.so (the reference's math headers compiled for the
host from the reference tree, see oracle/ref_kat.cpp) and evaluates it on
seeded inputs.  Run in the build container, where the reference tree is
mounted:

    python tests/golden/make_golden.py [<reference>/raytracer/include]

Without an argument the reference tree is $R2_REFERENCE_DIR.

The JSON holds inputs and reference outputs; tests/test_golden.py checks the
oracle's restatement against it without needing the reference.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ORACLE = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE, "_ref", "libr2ref.so")
OUT = os.path.join(HERE, "ref_math.json")


def build(ref_include: str) -> C.CDLL:
    subprocess.run(["make", "-s", "-C", ORACLE, "ref", f"REF={ref_include}"], check=True)
    lib = C.CDLL(LIB)
    P = C.c_void_p
    f = C.c_float
    lib.ref_u01.restype = f
    lib.ref_u01.argtypes = [f]
    lib.ref_fresnel.restype = f
    lib.ref_fresnel.argtypes = [f, f, f]
    lib.ref_warps.argtypes = [P, P]
    lib.ref_build_s.argtypes = [P, f, P]
    lib.ref_encode.argtypes = [P, P]
    lib.ref_decode.argtypes = [P, P]
    lib.ref_microfacet.argtypes = [f, f, f, f, P, P, P]
    lib.ref_microfacet_sample.argtypes = [f, f, f, f, P, P, P]
    lib.ref_ggx_sample_h.argtypes = [f, f, P, f, f, P]
    lib.ref_oren_nayar.argtypes = [f, P, P, P]
    lib.ref_oren_nayar_sample.argtypes = [f, P, P, P]
    lib.ref_frame.argtypes = [P, P, P]
    lib.ref_offset.argtypes = [P, P, P]
    lib.ref_sphere.argtypes = [P, f, P, P, P, f, P]
    lib.ref_find_interval.restype = C.c_int
    lib.ref_find_interval.argtypes = [P, C.c_int, f]
    lib.ref_sggx.argtypes = [P, P, P, P, f, f, P]
    lib.ref_sggx_sample.argtypes = [P, P, f, P, P, C.c_int, P]
    lib.ref_get_rotation.argtypes = [P, P]
    lib.ref_draws_used.restype = C.c_int
    lib.ref_vec3_arg_order.restype = C.c_int
    lib.ref_filter_scene.restype = C.c_int
    lib.ref_filter_scene.argtypes = [P, C.c_uint32, P, C.c_uint32, P, P, P, P, f, f]
    lib.ref_render_scene.restype = C.c_int
    lib.ref_render_scene.argtypes = [P, C.c_uint32, P, C.c_uint32, P, P, C.c_uint32, P, P, P, C.c_int, C.c_int]
    lib.ref_path_li.restype = C.c_int
    lib.ref_path_li.argtypes = [C.c_uint32, C.c_uint32, f, P, P, P, C.c_uint32, C.c_uint32, P, C.c_int, P]
    lib.ref_mesh_filter_voxel.restype = C.c_int
    lib.ref_mesh_filter_voxel.argtypes = [P] * 8 + [f, C.c_uint32, f, C.c_int, C.c_uint32, P, C.c_int, P]
    return lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _f32(x):
    return np.ascontiguousarray(x, np.float32)


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return _f32(v / np.linalg.norm(v, axis=1, keepdims=True))


# CMeshFilter::run cases: the mesh is rebuilt by the named seeded generator of
# renderer2_b200.scenes; the grid has `n` voxels along the longest extent.
MESH_FILTER_CASES = [
    dict(mesh="icosphere(2, 0.05, 1)", n=10, spv=64, iters=10, sigma_t=10.0, alpha=0.1, clip=1, seed=0,
         kd=(0.8, 0.6, 0.4), ks=(0.9, 0.9, 0.9), ggx=0.3, ior=1.5),
    dict(mesh="foliage(300, 3, 0.7, 5)", n=8, spv=128, iters=20, sigma_t=10.0, alpha=0.1, clip=1, seed=3,
         kd=(0.1, 0.6, 0.1), ks=(0.04, 0.04, 0.04), ggx=0.02, ior=1.33),
    dict(mesh="icosphere(1, 0.1, 7)", n=7, spv=48, iters=5, sigma_t=4.0, alpha=0.3, clip=0, seed=1,
         kd=(0.5, 0.5, 0.5), ks=(1.0, 1.0, 1.0), ggx=0.6, ior=1.2),
]


def curand_values_for(lib, u):
    """cuRAND values c with CSampler::uniformSample01(c) == u (float32), found next to u * (1 - FLT_EPSILON);
    NaN where no float maps to u exactly."""
    u = np.asarray(u, np.float32)
    eps = np.float32(2.0 ** -23)
    den = np.float32(np.float32(1.0) - eps) - np.float32(np.finfo(np.float32).tiny)
    base = (u.astype(np.float64) * float(den)).astype(np.float32)
    out = np.full(u.shape, np.nan, np.float32)
    for k in (0, 1, -1, 2, -2, 3, -3):
        c = np.nextafter(base, np.float32(np.inf) if k > 0 else np.float32(-np.inf)) if k else base
        for _ in range(abs(k) - 1):
            c = np.nextafter(c, np.float32(np.inf) if k > 0 else np.float32(-np.inf))
        got = np.clip((c / den).astype(np.float32) - np.finfo(np.float32).tiny, np.float32(0.0), np.float32(1.0) - eps)
        ok = np.isnan(out) & (got == u) & (c > 0)
        out[ok] = c[ok]
    zero = u == 0.0
    out[zero] = np.float32(1e-30)  # any c below FLT_MIN * den maps to 0
    for i in range(0, u.size, max(1, u.size // 64)):  # the numpy mapping agrees with the reference's own
        if not np.isnan(out.flat[i]):
            assert np.float32(lib.ref_u01(float(out.flat[i]))) == u.flat[i]
    return out


def mesh_filter_case(lib, mesh, n, spv, iters, sigma_t, alpha, clip, seed, kd, ks, ggx, ior):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    from renderer2_b200 import scenes
    m = eval("scenes." + mesh)
    m2w = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32)
    pos = np.ascontiguousarray(m.positions, np.float32)
    idx = np.ascontiguousarray(m.indices, np.uint32)
    nrm = np.ascontiguousarray(m.normals, np.float32)
    assert lib.ref_filter_scene(_p(pos), pos.shape[0], _p(idx), idx.shape[0], _p(nrm), _p(m2w), _p(_f32(kd)),
                                _p(_f32(ks)), ggx, ior) >= 0
    grid = O.setup_grid(pos.min(0), pos.max(0), m2w, scenes.voxel_size_for(m, n))
    nx, ny, nz = grid.num_voxels[:]
    order3 = lib.ref_vec3_arg_order()
    mats = [_f32(list(getattr(grid, k))) for k in ("index_to_model", "model_to_index", "model_to_world",
                                                    "world_to_model")]
    nv = np.array([nx, ny, nz], np.int32)
    bbmin, bbmax = _f32(list(grid.world_bb_min)), _f32(list(grid.world_bb_max))
    payload = np.zeros((nx * ny * nz, 32), np.uint8)
    inexact = 0
    s_idx = np.arange(spv, dtype=np.uint32)
    assert np.array_equal(np.array(scenes.philox4x32_10(3, 1, 0, 0, 17, seed)).ravel(), O.philox([3, 1, 0, 0], [17, seed]))
    for vid in range(nx * ny * nz):
        x, y, z = vid % nx, (vid // nx) % ny, vid // (nx * ny)
        r0 = np.stack(scenes.philox4x32_10(s_idx, 0, 0, 0, vid, seed), 1)  # the oracle's streams (voxel, seed)
        r1 = np.stack(scenes.philox4x32_10(s_idx, 1, 0, 0, vid, seed), 1)
        u = ((np.stack([r0[:, 0], r0[:, 1], r0[:, 2], r0[:, 3], r1[:, 0]], 1) >> 8).astype(np.float64)
             * (1.0 / 16777216.0)).astype(np.float32)
        if order3 == 1:  # glm::vec3(u(), u(), u()): the third component is drawn first in this build
            u[:, [0, 2]] = u[:, [2, 0]]
        c = curand_values_for(lib, u.reshape(-1))
        inexact += int(np.isnan(c).sum())
        c = np.where(np.isnan(c), np.float32(0.5), c).astype(np.float32)
        used = lib.ref_mesh_filter_voxel(_p(np.array([x, y, z], np.int32)), *[_p(a) for a in mats], _p(nv),
                                         _p(bbmin), _p(bbmax), sigma_t, iters, alpha, clip, spv, _p(c), c.size,
                                         _p(payload[vid]))
        assert used == 5 * spv, used
    return {"mesh": mesh, "n": n, "spv": spv, "iters": iters, "sigma_t": sigma_t, "alpha": alpha, "clip": clip,
            "seed": seed, "kd": list(kd), "ks": list(ks), "ggx": ggx, "ior": ior, "num_voxels": [nx, ny, nz],
            "draws_not_reproduced": inexact, "payload_hex": payload.tobytes().hex()}


# CPathIntegrator::Li case: two displaced icospheres (GGX 0.3 and 0.08) under a
# lognormal environment; one path per pixel, the draws of path k being
# path_draws(k) (Philox, key (k, PATH_KEY)); the reference has no depth limit
# below its 50 bounces.
PATH_CASES = [dict(room=False, width=24, height=20, fov=50.0, pos=(0.3, 0.6, 4.0), look_at=(0.4, 0.0, 0.0),
                   up=(0.0, 1.0, 0.0), env=(32, 16, 1.0, 9), draws=2 + 50 * 9),
              dict(room=True, width=24, height=20, fov=70.0, pos=(0.2, 0.4, 2.9), look_at=(0.4, 0.0, 0.0),
                   up=(0.0, 1.0, 0.0), env=(32, 16, 1.0, 9), draws=2 + 50 * 9)]
PATH_KEY = 77


def open_box(half=(3.0, 2.0, 3.0), n=4):
    """Floor, ceiling and three walls of a box (the +z side open), n x n quads each, normals facing in."""
    from renderer2_b200.filter import Mesh
    hx, hy, hz = half
    faces = [((0, -hy, 0), (1, 0, 0), (0, 0, 1), (0, 1, 0), (hx, hz)), ((0, hy, 0), (1, 0, 0), (0, 0, -1), (0, -1, 0), (hx, hz)),
             ((-hx, 0, 0), (0, 0, 1), (0, 1, 0), (1, 0, 0), (hz, hy)), ((hx, 0, 0), (0, 1, 0), (0, 0, 1), (-1, 0, 0), (hy, hz)),
             ((0, 0, -hz), (0, 1, 0), (1, 0, 0), (0, 0, 1), (hy, hx))]
    P, Nn, I = [], [], []
    for c, a, b, nrm, (ea, eb) in faces:
        c, a, b = np.asarray(c, float), np.asarray(a, float), np.asarray(b, float)
        g = np.linspace(-1.0, 1.0, n + 1)
        base = len(P)
        for j in range(n + 1):
            for i in range(n + 1):
                P.append(c + a * ea * g[i] + b * eb * g[j])
                Nn.append(nrm)
        for j in range(n):
            for i in range(n):
                v = base + j * (n + 1) + i
                I += [(v, v + 1, v + n + 2), (v, v + n + 2, v + n + 1)]
    return Mesh(_f32(P), np.asarray(I, np.uint32), _f32(Nn))


def path_scene(room=False):
    """(meshes as (mesh, kd, ks, ggx alpha, ior, translation)) of a Li case; the test rebuilds it."""
    sys.path.insert(0, ROOT)
    from renderer2_b200 import scenes
    spheres = [(scenes.icosphere(3, 0.05, 7), (0.7, 0.4, 0.2), (1.0, 1.0, 1.0), 0.3, 1.5, (0.0, 0.2, 0.0)),
               (scenes.icosphere(2, 0.1, 3), (0.2, 0.8, 0.3), (0.9, 0.9, 0.9), 0.08, 1.33, (1.6, 0.0, -0.5))]
    if not room:
        return spheres
    return spheres + [(open_box(), (0.85, 0.85, 0.8), (0.6, 0.6, 0.6), 0.5, 1.4, (0.0, 0.0, 0.0))]


def path_draws(k, n):
    """Uniforms k' / 2^24 of path k, as the oracle's 24-bit mapping produces them."""
    from renderer2_b200 import scenes
    i = np.arange(n, dtype=np.uint32)
    w = scenes.philox4x32_10(i, 0, 0, 0, k, PATH_KEY)[0]
    return ((w >> np.uint32(8)).astype(np.float64) * (1.0 / 16777216.0)).astype(np.float32)


def path_li_case(lib, c):
    sys.path.insert(0, ROOT)
    from renderer2_b200 import render_scenes as RS
    meshes = path_scene(c["room"])
    wpos, nrm, idx, tobj, m2w, mats = [], [], [], [], [], []
    base = 0
    for o, (m, kd, ks, a, ior, t) in enumerate(meshes):
        wpos.append(m.positions.astype(np.float32) + np.asarray(t, np.float32))
        nrm.append(m.normals.astype(np.float32))
        idx.append(m.indices.astype(np.uint32) + np.uint32(base))
        tobj.append(np.full(m.indices.shape[0], o, np.uint32))
        m2w.append(_f32([1, 0, 0, 0, 1, 0, 0, 0, 1, *t]))
        mats.append(_f32([*kd, *ks, a, ior]))
        base += m.positions.shape[0]
    wpos, nrm, idx = _f32(np.concatenate(wpos)), _f32(np.concatenate(nrm)), np.concatenate(idx)
    tobj, m2w, mats = np.concatenate(tobj), _f32(np.concatenate(m2w)), _f32(np.concatenate(mats))
    env = _f32(RS.lognormal_env(*c["env"]))
    assert lib.ref_render_scene(_p(wpos), wpos.shape[0], _p(idx), idx.shape[0], _p(nrm), _p(tobj), len(meshes),
                                _p(m2w), _p(mats), _p(env), env.shape[1], env.shape[0]) >= 0
    L = np.zeros((c["width"] * c["height"], 3), np.float32)
    used = np.zeros(c["width"] * c["height"], np.int32)
    inexact = 0
    for k in range(c["width"] * c["height"]):
        u = path_draws(k, c["draws"])
        cv = curand_values_for(lib, u)
        inexact += int(np.isnan(cv).sum())
        cv = np.where(np.isnan(cv), np.float32(0.5), cv).astype(np.float32)
        used[k] = lib.ref_path_li(c["width"], c["height"], c["fov"], _p(_f32(c["pos"])), _p(_f32(c["look_at"])),
                                  _p(_f32(c["up"])), k % c["width"], k // c["width"], _p(cv), cv.size, _p(L[k]))
    out = dict(c)
    out.update(key=PATH_KEY, draws_not_reproduced=inexact, draws_used=used.tolist(), L=L.tolist())
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.environ["R2_REFERENCE_DIR"], "raytracer", "include")
    lib = build(ref)
    rng = np.random.default_rng(20261203)
    g = {"vec2_arg_order": lib.ref_vec2_arg_order()}

    # cuRAND value -> uniformSample01
    cs = _f32(np.concatenate([rng.uniform(1e-7, 1.0, 64), [1.0, 0.5, 1e-7]]))
    g["u01"] = {"c": cs.tolist(), "u": [lib.ref_u01(float(c)) for c in cs]}

    # sampling warps, driven by two draws
    rows = []
    for _ in range(256):
        c = _f32(rng.uniform(1e-6, 1.0, 2))
        out = np.zeros(12, np.float32)
        lib.ref_warps(_p(c), _p(out))
        u = [lib.ref_u01(float(c[0])), lib.ref_u01(float(c[1]))]
        rows.append({"u": u, "out": out.tolist()})
    g["warps"] = rows

    rows = []
    for n, s in zip(unit(rng, 128), rng.uniform(0.0, 1.0, 128)):
        out = np.zeros(6, np.float32)
        lib.ref_build_s(_p(n), float(s), _p(out))
        rows.append({"n": n.tolist(), "sigma": float(s), "S": out.tolist()})
    g["build_s"] = rows

    rows = []
    for i in range(256):
        n = unit(rng, 1)[0]
        a = float(rng.uniform(0.02, 1.0))
        S = np.outer(n, n) + a * (np.eye(3) - np.outer(n, n))
        w = np.zeros(17, np.float32)
        w[0] = rng.lognormal(0, 2)
        w[1:7] = [S[0, 0], S[1, 1], S[2, 2], S[0, 1], S[0, 2], S[1, 2]]
        w[7:13] = rng.uniform(0, 1, 6)
        w[13:16] = unit(rng, 1)[0]
        w[16] = rng.uniform(1.0, 2.0)
        if i == 0:
            w[:] = 0.0
            w[16] = 1.0  # voxel without hits
        out = np.zeros(32, np.uint8)
        lib.ref_encode(_p(w), _p(out))
        dec = np.zeros(17, np.float32)
        lib.ref_decode(_p(out), _p(dec))
        rows.append({"in": w.tolist(), "bytes": out.tolist(), "decoded": dec.tolist()})
    g["payload"] = rows

    rows = []
    for _ in range(256):
        etaI, etaT = 1.0, float(rng.uniform(1.0, 2.5))
        c = float(rng.uniform(-1.0, 1.0))
        rows.append({"etaI": etaI, "etaT": etaT, "cos": c, "F": lib.ref_fresnel(etaI, etaT, c)})
    g["fresnel"] = rows

    def hemi(n, sign=1.0):
        v = unit(rng, n)
        v[:, 2] = np.abs(v[:, 2]) * sign
        return _f32(v)

    rows = []
    for wo, wi in zip(hemi(256), unit(rng, 256)):
        ax, ay = float(rng.uniform(0.05, 1.0)), float(rng.uniform(0.05, 1.0))
        etaT = float(rng.uniform(1.1, 2.0))
        out = np.zeros(2, np.float32)
        lib.ref_microfacet(ax, ay, 1.0, etaT, _p(wo), _p(wi), _p(out))
        c = _f32(rng.uniform(1e-6, 1.0, 2))
        so = np.zeros(5, np.float32)
        lib.ref_microfacet_sample(ax, ay, 1.0, etaT, _p(wo), _p(c), _p(so))
        h = np.zeros(3, np.float32)
        u1, u2 = float(rng.uniform(0, 1)), float(rng.uniform(0, 1))
        lib.ref_ggx_sample_h(ax, ay, _p(wo), u1, u2, _p(h))
        rows.append({"ax": ax, "ay": ay, "etaT": etaT, "wo": wo.tolist(), "wi": wi.tolist(), "f_pdf": out.tolist(),
                     "draw_u": [lib.ref_u01(float(c[0])), lib.ref_u01(float(c[1]))], "sample": so.tolist(),
                     "h_u": [u1, u2], "h": h.tolist()})
    g["microfacet"] = rows

    rows = []
    for wo, wi in zip(unit(rng, 256), unit(rng, 256)):
        r = float(rng.uniform(0.0, 1.0))
        out = np.zeros(2, np.float32)
        lib.ref_oren_nayar(r, _p(wo), _p(wi), _p(out))
        c = _f32(rng.uniform(1e-6, 1.0, 2))
        so = np.zeros(5, np.float32)
        lib.ref_oren_nayar_sample(r, _p(wo), _p(c), _p(so))
        rows.append({"roughness": r, "wo": wo.tolist(), "wi": wi.tolist(), "f_pdf": out.tolist(),
                     "draw_u": [lib.ref_u01(float(c[0])), lib.ref_u01(float(c[1]))], "sample": so.tolist()})
    g["oren_nayar"] = rows

    rows = []
    for n, v in zip(unit(rng, 128), unit(rng, 128)):
        out = np.zeros(9, np.float32)
        lib.ref_frame(_p(n), _p(v), _p(out))
        rows.append({"n": n.tolist(), "v": v.tolist(), "out": out.tolist()})
    g["frame"] = rows

    rows = []
    for _ in range(128):
        p = _f32(rng.uniform(-10, 10, 3))
        d = unit(rng, 1)[0]
        out = np.zeros(3, np.float32)
        lib.ref_offset(_p(p), _p(d), _p(out))
        rows.append({"p": p.tolist(), "d": d.tolist(), "out": out.tolist()})
    g["offset"] = rows

    rows = []
    for _ in range(256):
        c = _f32(rng.uniform(-1, 1, 3))
        r = float(rng.uniform(0.1, 2.0))
        o = _f32(c + rng.uniform(-1.5, 1.5, 3) * r)
        d = unit(rng, 1)[0]
        out = np.zeros(2, np.float32)
        nrm = _f32([0.0, 1.0, 0.0])
        lib.ref_sphere(_p(c), r, _p(nrm), _p(o), _p(d), 1e12, _p(out))
        rows.append({"c": c.tolist(), "r": r, "o": o.tolist(), "d": d.tolist(), "out": out.tolist()})
    g["sphere"] = rows

    rows = []
    for _ in range(128):
        n = int(rng.integers(2, 40))
        f = rng.uniform(0, 1, n - 1)
        cdf = _f32(np.concatenate([[0.0], np.cumsum(f) / f.sum()]))
        u = float(rng.uniform(0, 1))
        rows.append({"cdf": cdf.tolist(), "u": u, "k": lib.ref_find_interval(_p(cdf), n, u)})
    g["find_interval"] = rows

    rows = []
    for _ in range(128):
        n = unit(rng, 1)[0]
        a = float(rng.uniform(0.05, 1.0))
        S = np.outer(n, n) + a * (np.eye(3) - np.outer(n, n))
        S6 = _f32([S[0, 0], S[1, 1], S[2, 2], S[0, 1], S[0, 2], S[1, 2]])
        wo, wi = unit(rng, 1)[0], unit(rng, 1)[0]
        u1, u2 = float(rng.uniform(0, 1)), float(rng.uniform(0, 1))
        out = np.zeros(6, np.float32)
        lib.ref_sggx(_p(S6), _p(n), _p(wo), _p(wi), u1, u2, _p(out))
        rows.append({"S": S6.tolist(), "n": n.tolist(), "wo": wo.tolist(), "wi": wi.tolist(), "u": [u1, u2],
                     "out": out.tolist()})
    g["sggx"] = rows

    rows = []
    for _ in range(256):
        n = unit(rng, 1)[0]
        a = float(rng.uniform(0.05, 1.0))
        S = np.outer(n, n) + a * (np.eye(3) - np.outer(n, n))
        S6 = _f32([S[0, 0], S[1, 1], S[2, 2], S[0, 1], S[0, 2], S[1, 2]])
        wo = unit(rng, 1)[0]
        ior = float(rng.uniform(1.0, 3.0))
        c = _f32(rng.uniform(1e-6, 1.0, 5))
        out = np.zeros(4, np.float32)
        lib.ref_sggx_sample(_p(S6), _p(n), ior, _p(wo), _p(c), 5, _p(out))
        used = lib.ref_draws_used()
        rows.append({"S": S6.tolist(), "n": n.tolist(), "ior": ior, "wo": wo.tolist(),
                     "draw_u": [lib.ref_u01(float(x)) for x in c], "draws_used": used, "out": out.tolist()})
    g["sggx_sample"] = rows

    rows = []
    for n in [unit(rng, 1)[0] for _ in range(32)] + [_f32([0, 1, 0]), _f32([0, -1, 0]), _f32([1, 0, 0]),
                                                       _f32([0, 0, 1])]:
        out = np.zeros(16, np.float32)
        lib.ref_get_rotation(_p(n), _p(out))
        rows.append({"n": n.tolist(), "m": out.tolist()})
    g["get_rotation"] = rows

    g["vec3_arg_order"] = lib.ref_vec3_arg_order()
    g["mesh_filter"] = [mesh_filter_case(lib, **k) for k in MESH_FILTER_CASES]
    g["path_li"] = [path_li_case(lib, c) for c in PATH_CASES]

    with open(OUT, "w") as fh:
        json.dump(g, fh)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
