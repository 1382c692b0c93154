"""Benchmark of the Renderer2 hot paths on B200.

Headline (N=1 workload, config "surface path tracing"): 8x8 grid of displaced
icospheres (327,680 triangles, per-object GGX roughness U[0.05,1], albedo
U[0.2,0.9]) lit by a 512x256 lognormal(0,1.5) HDR environment, 1024x1024,
64 spp, max depth 8.  A step is one frame (64 spp in waves of several samples
per pixel, the wave size autotuned) over a device-resident scene; metric paths/s.

Second leg (config "filter at scale"): 500k leaf quads (1M tris) filtered to
256^3 with 256 samples/voxel and 20 iterations; metric filtered voxels/s,
reported in the "filter" object of the same line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference]

--impl reference times the CPU oracle port of the reference's integrator and
filter on the host cores (bounded samples of the same workloads).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_PATH = os.path.join(ROOT, "profiles", "traffic.json")
FALLBACK_HBM_GBS = 6650.0

RENDER_CFG = dict(width=1024, height=1024, spp=64, depth=8, seed=0)
FILTER_CFG = dict(n_quads=500_000, n_branches=20, clustered=0.7, seed=4, grid=256, spv=256, iters=20)
# Algorithmic bytes (SoA traffic a kernel must move; BVH nodes/triangles are
# excluded as L2-resident by design):
#   k_extend: queue id 4 + ray origin 16 + direction 16 + hit record 16 = 52 B per path segment
#   k_shadow_surfaces: record origin 16 + direction 16 + visibility 1 = 33 B per traced shadow ray
#   k_filter_sample: payload 32 + work-list id 4 = 36 B per filtered voxel
EXTEND_BYTES_PER_SEGMENT = 52.0
SHADOW_BYTES_PER_RAY = 33.0
FILTER_BYTES_PER_VOXEL = 36.0
# kernels of one BVH build + shading gather: bounds 2, Morton 1, radix sort 8 passes x 5, triangle gather 1,
# hierarchy 1, bottom-up 1, emission 1, shading gather 1
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # no measured FP32 figure on this pool
# media scenes:
#   extend phase (k_resolve rounds, k_track, k_collide): queue id 4 + ray in/out 64 + throughput in/out 32 + hit record 16 = 116 B per segment
#   shadow phase (k_shadow_resolve rounds, k_track): record origin 16 + direction 16 + tmax/medium 8 + queue id 4 + transmittance 4 = 48 B per slot
#   k_shade<true>: hit 16 + ray 32 + throughput 16 + radiance 16 + 2 records x 64 + continuation 48 = 256 B per segment
VOLUME_EXTEND_BYTES_PER_SEGMENT = 116.0
SHADOW_MEDIA_BYTES_PER_SLOT = 48.0
SHADE_BYTES_PER_SEGMENT = 256.0
VOLUME_CFG = dict(grid=256, n_quads=200_000, ico_subdiv=6, width=1920, height=1080, spp=16, depth=16, seed=0)
# one grid size per scene, 128^3 to 512^3 (config: "128^3-512^3")
VOLUME_BATCH_CFG = dict(scenes=16, grids=(128, 192, 256, 384, 512, 160, 224, 320, 128, 192, 256, 384, 144, 176, 208,
                                          288),
                        quads=(50_000, 150_000, 300_000), ico=(6, 7), width=1920, height=1080, spp=4, depth=16,
                        frame_spp=256)
SMALL_CFG = dict(grid=32, spv=64, iters=10, width=256, height=256, spp=16, depth=8)
SERVE_CFG = dict(jobs=60, rate=40.0, slots=4, budget=40 << 30, sizes=((256, 256), (384, 384), (512, 512), (1280, 720)),
                 spp=(4, 64), grids=(64, 96, 128, 192), quads=(10_000, 40_000, 100_000))
# the serving configuration's own mix (Poisson 20 req/s, 70 % renders 256^2..1920x1080 at spp log-uniform in
# [16, 1024], 30 % filters 64^3..512^3 over 20k..1M triangles, 150 GB budget), 30 jobs: `--case serving-stated`
SERVE_CFG_STATED = dict(jobs=30, rate=20.0, slots=6, budget=150 << 30,
                        sizes=((256, 256), (512, 512), (1280, 720), (1920, 1080)), spp=(16, 1024),
                        grids=(64, 128, 256, 512), quads=(10_000, 100_000, 500_000))
# forest leg: the forest generator's disc (radius 1000, 100,000 placement attempts) of three synthetic tree
# models, each filtered into 4 LODs; LODs chosen on the GPU for the generator's camera at 1920x1080
FOREST_CFG = dict(n_quads=20_000, grid=64, lods=4, attempts=100_000, radius=1000.0, width=1920, height=1080,
                  spp=4, depth=16, min_lod=0.0, covered_pixels=1.0, seed=0)


def _peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def _traffic(kernel: str):
    """DRAM bytes per work unit of a kernel from the committed ncu summary."""
    try:
        with open(TRAFFIC_PATH) as f:
            t = json.load(f)
        return t.get(kernel)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []  # (arrival time, line)
        self.window = None

    def start(self):
        """Starts nvidia-smi and waits (up to 10 s) for its first sample, so that it is sampling when the
        timed region begins."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 10.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def begin(self):
        self.window = [time.perf_counter(), None]

    def end(self):
        if self.window:
            self.window[1] = time.perf_counter()

    def stop(self):
        """Samples that arrived during the timed region (plus 0.3 s for the pipe); if the region was shorter
        than the sampling interval, the first sample after it began."""
        if not self.proc:
            return None
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        lines = [ln for _, ln in self.lines]
        if self.window and self.window[1] is not None:
            t0, t1 = self.window
            inside = [ln for t, ln in self.lines if t0 <= t <= t1 + 0.3]
            after = [ln for t, ln in self.lines if t >= t0]
            lines = inside or after[:1]
        sm, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


def _dist_setup():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def _max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"  # gloo groups reduce host tensors
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ------------------------------------------------------------------ workloads

def headline_config(world: int) -> dict:
    """The headline workload, printed identically by both arms."""
    c = RENDER_CFG
    return {"workload": "surface path tracing: 8x8 displaced icospheres (327,680 tris), 512x256 lognormal(0,1.5) env, "
                        "1024x1024, 64 spp, max depth 8; a step is the BVH build from the resident triangles + the "
                        "frame",
            "paths_per_step": c["width"] * c["height"] * c["spp"], "l2": "inputs + wave state larger than L2",
            "parallelism": f"replicas x{world}"}


def render_workload():
    from renderer2_b200 import render_scenes as RS
    from renderer2_b200 import raytracer as R
    desc, cam = RS.icosphere_grid_scene()
    c = RENDER_CFG
    cam = R.camera(c["width"], c["height"], 45.0, (0, 0, 24), (0, 0, 0), (0, 1, 0))
    prm = R.params(c["spp"], c["depth"], c["seed"])
    return desc, cam, prm


def filter_workload_params():
    from renderer2_b200 import filter as F
    c = FILTER_CFG
    return (F.params(samples_per_voxel=c["spv"], iterations=c["iters"]), None)


def filter_workload():
    from renderer2_b200 import filter as F
    from renderer2_b200 import scenes
    c = FILTER_CFG
    mesh = scenes.foliage(c["n_quads"], c["n_branches"], c["clustered"], c["seed"])
    mat = F.material(diffuse=(0.1, 0.6, 0.1), specular=(0.04, 0.04, 0.04), alpha=0.5, ior=1.5)
    prm = F.params(samples_per_voxel=c["spv"], iterations=c["iters"])
    vs = scenes.voxel_size_for(mesh, c["grid"])
    return mesh, mat, prm, vs


def _media_launches(tuning):
    """Kernel launches per bounce of a media scene: resolve, then per queued round track + resolve (the
    last one walking the rest), collide, events, shade, and the same rounds for the shadow rays, accum."""
    r = tuning.get("media_rounds") or 2
    return 6 + 4 * r


def _input_bytes(desc):
    b = desc["env"].nbytes
    for mesh, _, _ in desc["meshes"]:
        b += mesh.positions.nbytes + mesh.indices.nbytes + mesh.normals.nbytes
    return b


# ------------------------------------------------------------------ CPU baselines (oracle port)

def cpu_render_sample(desc, cam, prm, budget_s=15.0, threads=0):
    """Oracle paths/s on full-spp row bands at the frame centre; the oracle builds the scene's BVH in every call,
    so the time of a call over no pixels (the BVH build, done once per frame) is taken off each band."""
    import oracle_lib as O
    cores = threads or os.cpu_count() or 1
    W, H = cam.width, cam.height
    t0 = time.perf_counter()
    O.render(desc, cam, prm.spp, prm.max_depth, prm.seed, 0, 0, threads=cores, flags=prm.flags)
    t_build = time.perf_counter() - t0
    row = H // 2
    rows, done, t_work = 2, 0, 0.0
    while True:
        p0, p1 = row * W, min((row + rows) * W, W * H)
        t0 = time.perf_counter()
        O.render(desc, cam, prm.spp, prm.max_depth, prm.seed, p0, p1, threads=cores, flags=prm.flags)
        t_work += max(1e-6, time.perf_counter() - t0 - t_build)
        done += (p1 - p0)
        row += rows
        if t_work >= budget_s or row >= H:
            break
        rate = done / t_work
        rows = max(1, min(int((budget_s - t_work) * rate / W), 4 * rows, H - row))
    paths = done * prm.spp
    return {"value": paths / t_work, "unit": "paths/s", "cores": cores, "kind": "port", "seconds": t_work,
            "bvh_build_s": t_build,
            "sample": f"{done // W} rows x {W} px x {prm.spp} spp at the frame centre ({paths} paths), "
                      f"the BVH build ({t_build:.2f} s, once per frame) taken off each band"}


def ref_code_render_sample(desc, cam, prm, budget_s=10.0, threads=0):
    """The reference's own CPathIntegrator::Li, compiled for the host (oracle/_ref/libr2ref.so, built from the
    reference's sources; the scene's closest hits come from the oracle's BVH and the environment from the
    oracle's map), timed on full-spp row bands at the frame centre.  Its bounce cap is its own 50 (Russian
    roulette from bounce 4), not the configuration's depth.  None when the library was not built."""
    import ctypes as C
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle", "_ref", "libr2ref.so")
    if not os.path.exists(path) or desc.get("media") or desc.get("shapes"):
        return None
    lib = C.CDLL(path)
    P = C.c_void_p
    lib.ref_render_scene.argtypes = [P, C.c_uint32, P, C.c_uint32, P, P, C.c_uint32, P, P, P, C.c_int, C.c_int]
    lib.ref_render_paths.argtypes = [C.c_uint32, C.c_uint32, C.c_float, P, P, P, C.c_uint32, C.c_uint32, C.c_uint32,
                                     C.c_uint32, P, C.c_int]
    from renderer2_b200 import render_scenes as RS
    wpos, _ = RS.world_vertices(desc)
    nrm, idx, tobj, m2w, mats = [], [], [], [], []
    base = 0
    for o, entry in enumerate(desc["meshes"]):
        mesh, mat, t = entry[:3]
        nrm.append(np.asarray(mesh.normals, np.float32))
        idx.append(np.asarray(mesh.indices, np.uint32) + np.uint32(base))
        tobj.append(np.full(mesh.indices.shape[0], o, np.uint32))
        m2w.append(np.asarray(t, np.float32))
        mats.append(np.array([*mat.diffuse, *mat.specular, mat.alpha_x, mat.eta_t], np.float32))
        base += mesh.positions.shape[0]
    arrs = [np.ascontiguousarray(a) for a in (wpos, np.concatenate(nrm), np.concatenate(idx), np.concatenate(tobj),
                                              np.concatenate(m2w), np.concatenate(mats))]
    wp, nr, ix, to, mw, ma = arrs
    env = np.ascontiguousarray(desc["env"], np.float32)
    assert lib.ref_render_scene(wp.ctypes.data, wp.shape[0], ix.ctypes.data, ix.shape[0], nr.ctypes.data,
                                to.ctypes.data, len(desc["meshes"]), mw.ctypes.data, ma.ctypes.data, env.ctypes.data,
                                env.shape[1], env.shape[0]) >= 0
    cores = threads or os.cpu_count() or 1
    W, H = cam.width, cam.height
    f3 = lambda v: np.ascontiguousarray(v, np.float32)  # noqa: E731
    pos, look, up = f3(cam.pos[:]), f3(cam.look_at[:]), f3(cam.up[:])
    row, rows, done, t_work = H // 2, 2, 0, 0.0
    while True:
        p0, p1 = row * W, min((row + rows) * W, W * H)
        out = np.zeros((p1 - p0, 3), np.float32)
        t0 = time.perf_counter()
        assert lib.ref_render_paths(W, H, cam.fov_deg, pos.ctypes.data, look.ctypes.data, up.ctypes.data, prm.spp,
                                    prm.seed, p0, p1, out.ctypes.data, cores) == 0
        t_work += time.perf_counter() - t0
        done += p1 - p0
        row += rows
        if t_work >= budget_s or row >= H:
            break
        rows = max(1, min(int((budget_s - t_work) * done / t_work / W), 4 * rows, H - row))
    paths = done * prm.spp
    return {"value": paths / t_work, "unit": "paths/s", "cores": cores, "kind": "reference", "seconds": t_work,
            "sample": f"{done // W} rows x {W} px x {prm.spp} spp at the frame centre ({paths} paths) through the "
                      "reference's CPathIntegrator::Li compiled for the host (bounce cap 50, its own)"}


def ref_code_filter_sample(mesh, mat, prm, vs, budget_s=10.0, threads=0):
    """The reference's own CMeshFilter::run with estimateDensity, compiled for the host (oracle/_ref/libr2ref.so;
    closest hits from the oracle's BVH), on contiguous z-slices at the grid centre.  None when not built."""
    import ctypes as C
    import oracle_lib as O
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle", "_ref", "libr2ref.so")
    if not os.path.exists(path) or prm.samples_per_voxel > 1000:
        return None
    lib = C.CDLL(path)
    P = C.c_void_p
    lib.ref_filter_scene.argtypes = [P, C.c_uint32, P, C.c_uint32, P, P, P, P, C.c_float, C.c_float]
    lib.ref_filter_voxels.argtypes = [P, P, P, P, P, P, P, C.c_float, C.c_uint32, C.c_float, C.c_int, C.c_uint32,
                                      C.c_uint32, C.c_uint64, C.c_uint64, P, C.c_int]
    m2w = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32)
    pos = np.ascontiguousarray(mesh.positions, np.float32)
    idx = np.ascontiguousarray(mesh.indices, np.uint32)
    nrm = np.ascontiguousarray(mesh.normals, np.float32)
    kd = np.ascontiguousarray(mat.diffuse[:], np.float32)
    ks = np.ascontiguousarray(mat.specular[:], np.float32)
    t0 = time.perf_counter()
    assert lib.ref_filter_scene(pos.ctypes.data, pos.shape[0], idx.ctypes.data, idx.shape[0], nrm.ctypes.data,
                                m2w.ctypes.data, kd.ctypes.data, ks.ctypes.data, mat.alpha_x, mat.eta_t) >= 0
    t_build = time.perf_counter() - t0
    g = O.setup_grid(pos.min(0), pos.max(0), m2w, vs)
    nx, ny, nz = g.num_voxels[:]
    mats = [np.ascontiguousarray(list(getattr(g, k)), np.float32)
            for k in ("index_to_model", "model_to_index", "model_to_world", "world_to_model")]
    nv = np.array([nx, ny, nz], np.int32)
    bbmin = np.ascontiguousarray(list(g.world_bb_min), np.float32)
    bbmax = np.ascontiguousarray(list(g.world_bb_max), np.float32)
    cores = threads or os.cpu_count() or 1
    slab = nx * ny
    z, done, t_work, nsl = nz // 2, 0, 0.0, 1
    while True:
        v0, v1 = z * slab, min((z + nsl) * slab, nx * ny * nz)
        out = np.zeros((v1 - v0, 32), np.uint8)
        t0 = time.perf_counter()
        assert lib.ref_filter_voxels(*[a.ctypes.data for a in mats], nv.ctypes.data, bbmin.ctypes.data,
                                     bbmax.ctypes.data, prm.sigma_t, prm.estimation_iterations, prm.alpha,
                                     int(prm.clip_rays), prm.samples_per_voxel, prm.seed, v0, v1, out.ctypes.data,
                                     cores) == 0
        t_work += time.perf_counter() - t0
        done += v1 - v0
        z += nsl
        if t_work >= budget_s or z >= nz:
            break
        nsl = max(1, min(int((budget_s - t_work) * (done / t_work) / slab), 4 * nsl, nz - z))
    return {"value": done / t_work, "unit": "voxels/s", "cores": cores, "kind": "reference", "seconds": t_work,
            "sample": f"{done // slab} z-slices of {nx}x{ny} at the grid centre, {prm.samples_per_voxel} spv, through "
                      f"the reference's CMeshFilter::run compiled for the host (BVH build {t_build:.2f}s excluded)"}


def cpu_render_baseline(desc, cam, prm, budget_s=15.0):
    """The CPU baseline of a render: the reference's own integrator compiled for the host where it was built
    (surface scenes), else the oracle port."""
    r = ref_code_render_sample(desc, cam, prm, budget_s=budget_s)
    return r if r is not None else cpu_render_sample(desc, cam, prm, budget_s=budget_s)


def cpu_filter_sample(mesh, mat, prm, vs, budget_s=15.0, threads=0, keep=None):
    """Oracle voxels/s on contiguous z-slices at the grid centre (BVH build subtracted).  keep (a dict):
    receives the first slab's voxel range and the oracle's FP64 records of it ("v0", "v1", "wide")."""
    import oracle_lib as O
    from renderer2_b200 import _native as N
    m2w = N.identity43()
    g = O.setup_grid(mesh.positions.min(0).astype(np.float32), mesh.positions.max(0).astype(np.float32), m2w, vs)
    nx, ny, nz = g.num_voxels[:]
    slab = nx * ny
    cores = threads or os.cpu_count() or 1
    t0 = time.perf_counter()
    O.filter_voxels(mesh, O.material_from(mat), m2w, g, O.params_from(prm), 0, 0, 0, cores)
    t_build = time.perf_counter() - t0
    z, done, t_work, nsl = nz // 2, 0, 0.0, 1
    while True:
        v0, v1 = z * slab, min((z + nsl) * slab, nx * ny * nz)
        t0 = time.perf_counter()
        ow, _ = O.filter_voxels(mesh, O.material_from(mat), m2w, g, O.params_from(prm), v0, v1, 0, cores)
        t_work += max(time.perf_counter() - t0 - t_build, 1e-9)
        if keep is not None and "wide" not in keep:
            keep.update(v0=v0, v1=v1, wide=ow)
        done += v1 - v0
        z += nsl
        if t_work >= budget_s or z >= nz:
            break
        nsl = max(1, min(int((budget_s - t_work) * (done / t_work) / slab), nz - z))
    return {"value": done / t_work, "unit": "voxels/s", "cores": cores, "kind": "port",
            "sample": f"{done // slab} z-slices of {nx}x{ny} at the grid centre, {FILTER_CFG['spv']} spv, "
                      f"BVH build ({t_build:.2f}s) excluded"}


# ------------------------------------------------------------------ native legs

def filter_accuracy(gw, gh, ow):
    """Largest relative errors of the FP32 records (gw) and the FP16 payload (gh) against the oracle's FP64 ones
    (ow) over the voxels with hits: density relative to itself, S entries relative to the voxel's largest
    diagonal entry."""
    h = (ow[:, 17] > 0) & np.isfinite(ow[:, 0])
    scale = np.max(np.abs(ow[h, 1:4]), axis=1, keepdims=True)
    out = {"voxels_compared": int(h.sum()), "hits_bit_exact": bool(np.array_equal(gw[:, 17], ow[:, 17]))}
    for name, rec in (("fp32", gw), ("fp16", gh)):
        out[name] = {"density": float((np.abs(rec[h, 0] - ow[h, 0]) / np.abs(ow[h, 0])).max(initial=0.0)),
                     "S": float((np.abs(rec[h, 1:7] - ow[h, 1:7]) / scale).max(initial=0.0))}
    return out


def gpu_filter_records(sc, g, prm, v0, v1):
    """FP32 records and FP16 payloads of voxels [v0, v1) from one untimed GPU pass."""
    import torch
    nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
    out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    wide = torch.empty(nvox * 20, dtype=torch.float32, device="cuda")
    f16 = torch.empty(nvox * 8, dtype=torch.float16, device="cuda")
    sc.run(g, prm, out.data_ptr(), wide.data_ptr(), f16.data_ptr())
    torch.cuda.synchronize()
    gw = wide.view(nvox, 20)[v0:v1].cpu().numpy().astype(np.float64)
    gh = f16.view(nvox, 8)[v0:v1].cpu().numpy().astype(np.float64)
    return gw, gh


def bench_render(args, world, local):
    import torch
    from renderer2_b200 import raytracer as R
    from renderer2_b200 import render_scenes as RS
    desc, cam, prm = render_workload()
    sc = RS.build_scene(desc)
    tuning = sc.autotune(cam, prm).as_dict()  # set-up: launch tuning of this frame (never changes the image)
    npix = cam.width * cam.height
    frame = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(args.warmup):
        sc.render_device(cam, prm, frame.data_ptr(), stream)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    _barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    st = np.zeros(8)
    stats = []
    evb = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
            torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks.begin()
    ev0.record()
    for k in range(args.steps):
        # one step = BVH build from the resident triangles + the frame (config "BVH build + trace");
        # inputs (BVH 21 MB nodes + 16 MB tris + state ~200 MB per wave) exceed L2; no flush needed
        evb[k][0].record()
        sc.rebuild(stream)
        evb[k][1].record()
        sc.render_device(cam, prm, frame.data_ptr(), stream, stats=st)
        evb[k][2].record()
        stats.append(st.copy())
    ev1.record()
    torch.cuda.synchronize()
    clocks.end()
    _barrier(world)
    ck = clocks.stop()
    total_ms = _max_over_ranks(ev0.elapsed_time(ev1), world)
    build_ms = float(np.median([a.elapsed_time(b) for a, b, _ in evb]))
    latency = step_latency([a.elapsed_time(c) for a, _, c in evb])
    paths = npix * prm.spp
    value = world * paths * args.steps / (total_ms / 1e3)
    st = np.mean(np.array(stats), axis=0)
    seg, shadow = st[2], st[3]
    ms_wave = {"extend": st[4], "shade": st[5], "shadow": st[6], "accum": st[7]}
    # dominant kernel over the frame; a wave renders S samples of every pixel
    S = sc.wave_samples(cam, prm)
    seg_wave, sh_wave = seg * S / prm.spp, shadow * S / prm.spp
    dom = "extend" if ms_wave["extend"] >= ms_wave["shadow"] else "shadow"
    peak, peak_kind = _peaks()
    if dom == "extend":
        alg = EXTEND_BYTES_PER_SEGMENT * seg_wave
        kname = "k_extend"
    else:
        alg = SHADOW_BYTES_PER_RAY * sh_wave
        kname = "k_shadow_surfaces"
    kms = ms_wave[dom]
    launches = prm.max_depth
    achieved = alg / (kms / 1e3) / 1e9
    tr = _traffic(kname)
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": (tr["bytes_per_unit"] * (seg_wave if dom == "extend" else sh_wave) / launches)
                if tr else None,
                "alg_bytes_per_launch": alg / launches, "avg_launch_ms": kms / launches,
                "samples_per_wave": S,
                "note": "per-launch figures averaged over the bounces of the timed middle wave; "
                        "traversal is L2/issue bound, see rays_per_s",
                "rays_per_s": (seg + shadow) / (st[1] / 1e3), "kernel_ms_per_wave": ms_wave}
    # end to end through the C ABI with host buffers, every step: the frame's world-space vertices and normals
    # copied from pinned host memory (r2_scene_set_vertices), the BVH rebuilt (r2_scene_rebuild), the frame
    # rendered and copied to a pinned host buffer (r2_render_host, which waits for it)
    pos, nrm = RS.world_vertices(desc)
    hpos = torch.from_numpy(pos).pin_memory()
    hnrm = torch.from_numpy(nrm).pin_memory()
    hframe = torch.empty(npix * 3, dtype=torch.float32).pin_memory()
    nv = pos.shape[0]

    def e2e_step():
        sc.set_vertices(hpos.data_ptr(), hnrm.data_ptr(), nverts=nv)
        sc.rebuild()
        sc.render(cam, prm, out_ptr=hframe.data_ptr())

    e2e_step()  # warm-up (first use of the host frame buffer)
    e2e_ms = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_step()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = _max_over_ranks(float(np.median(e2e_ms)), world)
    bvh_nodes, bvh_height, bvh_launches = sc.bvh_info()
    e2e = {"value": world * paths / (e2e_ms / 1e3), "unit": "paths/s", "h2d_bytes_per_step": int(pos.nbytes + nrm.nbytes),
           "d2h_bytes_per_step": int(npix * 12), "ms_per_step": e2e_ms,
           "calls": "r2_scene_set_vertices (pinned) + r2_scene_rebuild + r2_render_host (pinned frame)"}
    sc.close()
    # cold start for reference: a new scene from the arrays (upload, BVH, default launch tuning) and one frame
    t0 = time.perf_counter()
    s2 = RS.build_scene(desc)
    t1 = time.perf_counter()
    s2.render(cam, prm)
    t2 = time.perf_counter()
    s2.close()
    e2e["cold_start"] = {"value": world * paths / (t2 - t0), "scene_build_ms": (t1 - t0) * 1e3,
                         "render_and_download_ms": (t2 - t1) * 1e3, "h2d_bytes": int(_input_bytes(desc))}
    sort_launches = 4 * (prm.max_depth - 1) if tuning.get("sort_rays") else 0  # ray sort before bounces 1..
    launches_per_step = (prm.spp // S) * (2 + 4 * prm.max_depth + sort_launches) + bvh_launches
    return dict(value=value, total_ms=total_ms, roofline=roofline, e2e=e2e, clocks=ck, paths=paths, tuning=tuning,
                latency=latency,
                segments_per_frame=seg, shadow_rays_per_frame=shadow, launches=launches_per_step * args.steps,
                bvh_build_ms=build_ms, render_ms=total_ms / args.steps - build_ms, desc=desc, cam=cam, prm=prm,
                bvh={"method": "Karras" if R.bvh_method() == R.BVH_KARRAS else "PLOC", "inner_nodes": bvh_nodes,
                     "height": bvh_height, "build_launches": bvh_launches})


def bench_filter(args, world, local, grid=None, steps=None, warmup=None, e2e_run=True, mesh_mat=None):
    """Filter at scale (500k leaf quads, 256 spv, 20 iterations) on the 256^3 grid, or `grid`^3."""
    import torch
    from renderer2_b200 import filter as F
    from renderer2_b200 import scenes
    mesh, mat, prm, vs = filter_workload() if mesh_mat is None else (mesh_mat + filter_workload_params())
    if grid is not None:
        vs = scenes.voxel_size_for(mesh, grid)
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    sc = F.FilterScene(mesh, mat)
    g = sc.grid(vs)
    nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
    out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = np.zeros(3)
    for _ in range(warmup):
        flush.fill_(1)
        sc.run(g, prm, out.data_ptr(), stream=stream, stats=st)
    torch.cuda.synchronize()
    _barrier(world)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    step_ms, kernel_ms, cand, per_step = 0.0, [], [], []
    for _ in range(steps):
        flush.fill_(1)  # 256 MiB write evicts L2 between steps
        ev0.record()
        sc.run(g, prm, out.data_ptr(), stream=stream, stats=st)
        ev1.record()
        torch.cuda.synchronize()
        per_step.append(ev0.elapsed_time(ev1))
        step_ms += per_step[-1]
        kernel_ms.append(st[2])
        cand.append(st[1])
    _barrier(world)
    total_ms = _max_over_ranks(step_ms, world)
    value = world * nvox * steps / (total_ms / 1e3)
    h2d = mesh.positions.nbytes + mesh.indices.nbytes + mesh.normals.nbytes
    del out, flush
    # the central z-slice's FP32 records and FP16 payloads (untimed), for the accuracy against the oracle
    nx, ny, nz = g.num_voxels[:]
    slab = (nz // 2 * nx * ny, (nz // 2 + 1) * nx * ny)
    gpu_slab = gpu_filter_records(sc, g, prm, *slab)
    e2e = None
    if e2e_run:
        # end to end: r2_filter_mesh with the mesh in host memory and the payloads copied into a pinned host
        # buffer (upload, BVH build, classification, sampling, download, every step)
        hout = torch.empty(nvox * 32, dtype=torch.uint8).pin_memory()
        e2e_ms = []
        for k in range(6):  # the median of five calls: host-side scene set-up varies from call to call
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            F.filter_mesh(mesh, mat, prm, vs, out_ptr=hout.data_ptr(), out_capacity=nvox)
            if k:  # the first call warms the host buffer and the device allocations
                e2e_ms.append((time.perf_counter() - t0) * 1e3)
        e2e_ms = _max_over_ranks(float(np.median(e2e_ms)), world)
        del hout
        e2e = {"value": world * nvox / (e2e_ms / 1e3), "unit": "voxels/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(nvox * 32), "ms_per_step": e2e_ms}
    kms = float(np.mean(kernel_ms))
    peak, peak_kind = _peaks()
    alg = FILTER_BYTES_PER_VOXEL * nvox
    achieved = alg / (kms / 1e3) / 1e9
    tr = _traffic("k_filter_sample")
    rays = float(np.mean(cand)) * FILTER_CFG["spv"]
    # arithmetic figure from the counting build of the same kernel (untimed):
    # 24 FLOPs per inner node visited, 30 per triangle tested, 40 per ray
    cnt_out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    n_rays, n_nodes, n_tris = sc.count(g, prm, cnt_out.data_ptr())
    del cnt_out
    flops = 24.0 * n_nodes + 30.0 * n_tris + 40.0 * n_rays
    fp32_peak = FP32_NOMINAL_TFLOPS
    sc.close()
    n = grid or FILTER_CFG["grid"]
    return {"metric": "filtered voxels/s", "value": value, "unit": "voxels/s", "ms_per_step": total_ms / steps,
            "steps": steps,
            "config": {"workload": f"filter at scale: 500k leaf quads (1M tris), {n}^3, 256 spv, 20 iters",
                       "voxels": nvox, "candidate_voxels": float(np.mean(cand)),
                       "l2": "256 MiB flush write between steps"},
            "latency": step_latency(per_step),
            "roofline": {"bound": "hbm", "kernel": "k_filter_sample", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": tr["bytes_per_unit"] * nvox if tr else None,
                         "kernel_ms": kms, "rays_per_s": rays / (kms / 1e3),
                         "note": "36 B/voxel algorithmic; bound by issue (triangle tests, density fit) and L2 latency",
                         "fp32": {"achieved": flops / (kms / 1e3) / 1e12, "peak": fp32_peak, "unit": "TFLOP/s",
                                  "frac": flops / (kms / 1e3) / 1e12 / fp32_peak,
                                  "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 2 x 1.965 GHz",
                                  "flops_per_launch": flops, "rays": n_rays, "inner_nodes_visited": n_nodes,
                                  "triangles_tested": n_tris,
                                  "formula": "24 per inner node visited + 30 per triangle tested + 40 per ray"}},
            "e2e": e2e,
            "gpu_launches": 2 * steps, "_mesh": (mesh, mat, prm, vs), "_gpu_slab": (slab, gpu_slab)}


def surface_roofline(st, S, spp, launches):
    """HBM roofline of the dominant surface traversal kernel from r2_render_device's stats of a frame: per-wave
    kernel times, segments and shadow rays of the frame, S samples per wave."""
    seg_wave, sh_wave = st[2] * S / spp, st[3] * S / spp
    ext, shd = st[4], st[6]
    dom_ext = ext >= shd
    alg = EXTEND_BYTES_PER_SEGMENT * seg_wave if dom_ext else SHADOW_BYTES_PER_RAY * sh_wave
    kms = ext if dom_ext else shd
    peak, kind = _peaks()
    achieved = alg / (kms / 1e3) / 1e9
    return {"bound": "hbm", "kernel": "k_extend" if dom_ext else "k_shadow_surfaces", "achieved": achieved,
            "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": kind,
            "alg_bytes_per_launch": alg / launches, "avg_launch_ms": kms / launches, "samples_per_wave": S}


def bench_small(args, world, local):
    """Plain method, small: icosphere subdivision 4 (5,120 triangles) displaced by value noise 0.05, GGX
    roughness 0.3, albedo 0.8; SGGX filter to 32^3 (64 spv, 10 iterations) and a 256x256 frame (16 spp, depth
    8, constant white environment).  A step filters the grid and renders the frame (BVH build from the resident
    triangles + trace), on resident scenes; each part is timed on the stream."""
    import torch
    import oracle_lib as O
    from renderer2_b200 import filter as F
    from renderer2_b200 import raytracer as R
    from renderer2_b200 import render_scenes as RS
    from renderer2_b200 import scenes
    c = SMALL_CFG
    desc, cam = RS.icosphere_scene()
    mesh, mat, m2w = desc["meshes"][0]
    fprm = F.params(samples_per_voxel=c["spv"], iterations=c["iters"])
    fsc = F.FilterScene(mesh, mat)
    g = fsc.grid(scenes.voxel_size_for(mesh, c["grid"]))
    nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
    out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    sc = RS.build_scene(desc)
    prm = R.params(c["spp"], c["depth"], 0)
    tuning = sc.autotune(cam, prm).as_dict()
    npix = cam.width * cam.height
    frame = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    fst, rst = np.zeros(3), np.zeros(8)
    for _ in range(args.warmup):
        fsc.run(g, fprm, out.data_ptr(), stream=stream)
        sc.rebuild(stream)
        sc.render_device(cam, prm, frame.data_ptr(), stream)
    torch.cuda.synchronize()
    _barrier(world)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    fk, rs = [], []
    for k in range(args.steps):
        ev[k][0].record()
        fsc.run(g, fprm, out.data_ptr(), stream=stream, stats=fst)
        ev[k][1].record()
        sc.rebuild(stream)
        sc.render_device(cam, prm, frame.data_ptr(), stream, stats=rst)
        ev[k][2].record()
        fk.append(fst[2])
        rs.append(rst.copy())
    torch.cuda.synchronize()
    _barrier(world)
    f_ms = _max_over_ranks(sum(e[0].elapsed_time(e[1]) for e in ev), world)
    r_ms = _max_over_ranks(sum(e[1].elapsed_time(e[2]) for e in ev), world)
    paths = npix * c["spp"]
    S = sc.wave_samples(cam, prm)
    rst = np.mean(np.array(rs), axis=0)
    peak, kind = _peaks()
    kms = float(np.mean(fk))
    fachieved = FILTER_BYTES_PER_VOXEL * nvox / (kms / 1e3) / 1e9
    # end to end, host buffers: the filter through r2_filter_mesh into pinned memory; the frame through the
    # vertex upload from pinned memory, the BVH rebuild and r2_render_host into pinned memory
    hv = torch.empty(nvox * 32, dtype=torch.uint8).pin_memory()
    pos, nrm = RS.world_vertices(desc)
    hp, hn = torch.from_numpy(pos).pin_memory(), torch.from_numpy(nrm).pin_memory()
    hf = torch.empty(npix * 3, dtype=torch.float32).pin_memory()

    def e2e_step():
        F.filter_mesh(mesh, mat, fprm, scenes.voxel_size_for(mesh, c["grid"]), out_ptr=hv.data_ptr(),
                      out_capacity=nvox)
        sc.set_vertices(hp.data_ptr(), hn.data_ptr(), nverts=pos.shape[0])
        sc.rebuild()
        sc.render(cam, prm, out_ptr=hf.data_ptr())

    e2e_step()
    e2e_ms = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_step()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = _max_over_ranks(float(np.median(e2e_ms)), world)
    bvh_launches = sc.bvh_info()[2]
    # accuracy at this configuration: the whole grid against the FP64 oracle, the frame against the oracle's
    gw, gh = gpu_filter_records(fsc, g, fprm, 0, nvox)
    acc, cpu = None, None
    gframe = hf.numpy().reshape(-1, 3).copy()
    if world == 1:
        t0 = time.perf_counter()
        ow, _ = O.filter_voxels(mesh, O.material_from(mat), m2w, O.grid_from(g), O.params_from(fprm))
        t_f = time.perf_counter() - t0
        t0 = time.perf_counter()
        of = O.render(desc, cam, c["spp"], c["depth"], 0)
        t_r = time.perf_counter() - t0
        rel = (np.abs(gframe - of) / np.maximum(1.0, np.abs(of))).max(axis=1)
        acc = {"filter": filter_accuracy(gw, gh, ow),
               "frame_pixels_within_1e-4_of_oracle": float((rel <= 1e-4).mean())}
        cores = os.cpu_count() or 1
        cpu = {"filter": {"value": nvox / t_f, "unit": "voxels/s", "cores": cores, "kind": "port",
                          "sample": f"the whole {c['grid']}^3 grid (BVH build included)"},
               "render": {"value": paths / t_r, "unit": "paths/s", "cores": cores, "kind": "port",
                          "sample": f"the whole {cam.width}x{cam.height} frame at {c['spp']} spp (BVH build included)"}}
    fsc.close()
    sc.close()
    total_ms = f_ms + r_ms
    return {"metric": "filtered voxels/s; paths/s", "value": world * nvox * args.steps / (f_ms / 1e3),
            "unit": "voxels/s", "paths_per_s": world * paths * args.steps / (r_ms / 1e3),
            "ms_per_step": total_ms / args.steps, "filter_ms_per_step": f_ms / args.steps,
            "render_ms_per_step": r_ms / args.steps,
            "config": {"workload": "plain method, small: icosphere subdivision 4 (5,120 tris) displaced 0.05, GGX 0.3 "
                                   "albedo 0.8; SGGX filter to 32^3, 64 spv, 10 iterations; 256x256, 16 spp, depth 8, "
                                   "constant white environment", "voxels": nvox, "paths_per_step": paths,
                       "tuning": tuning, "l2": "small inputs: L2-resident (reported as such)"},
            "roofline": {"filter": {"bound": "hbm", "kernel": "k_filter_sample", "achieved": fachieved, "peak": peak,
                                    "unit": "GB/s", "frac": fachieved / peak, "peak_source": kind,
                                    "kernel_ms": kms},
                         "render": surface_roofline(rst, S, c["spp"], c["depth"])},
            "e2e": {"value": world * nvox / (e2e_ms / 1e3), "unit": "voxels/s",
                    "paths_per_s": world * paths / (e2e_ms / 1e3), "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": int(mesh.positions.nbytes + mesh.indices.nbytes + mesh.normals.nbytes
                                              + pos.nbytes + nrm.nbytes),
                    "d2h_bytes_per_step": int(nvox * 32 + npix * 12)},
            "accuracy": acc, "cpu_baseline": cpu,
            "gpu_launches": (2 + bvh_launches + (c["spp"] // S) * (2 + 4 * c["depth"] + (
                4 * (c["depth"] - 1) if tuning.get("sort_rays") else 0))) * args.steps}


def media_roofline(st, S, spp, depth):
    """HBM roofline of the dominant phase of a media frame from its render statistics st (the 8 values of
    r2_render_device) and S samples per wave."""
    ms_wave = {"extend": st[4], "shade": st[5], "shadow": st[6], "accum": st[7]}
    seg_wave = st[2] * S / spp
    dom = max(("extend", "shadow", "shade"), key=lambda k: ms_wave[k])
    per_unit = {"extend": (VOLUME_EXTEND_BYTES_PER_SEGMENT, seg_wave, "extend phase"),
                "shadow": (SHADOW_MEDIA_BYTES_PER_SLOT, 2.0 * seg_wave, "shadow phase"),
                "shade": (SHADE_BYTES_PER_SEGMENT, seg_wave, "k_shade<true>")}[dom]
    alg = per_unit[0] * per_unit[1]
    kms = ms_wave[dom]
    peak, peak_kind = _peaks()
    achieved = alg / (kms / 1e3) / 1e9
    tr = _traffic(per_unit[2])
    return {"bound": "hbm", "kernel": per_unit[2], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind,
            "traffic": tr["bytes_per_unit"] * per_unit[1] / depth if tr else None,
            "alg_bytes_per_launch": alg / depth, "avg_launch_ms": kms / depth,
            "note": "delta/ratio tracking is latency bound on dependent grid lookups",
            "kernel_ms_per_wave": ms_wave}


def step_latency(ms):
    """p50 / p99 of per-step device times (ms)."""
    a = np.asarray(ms, np.float64)
    return {"p50_ms": float(np.percentile(a, 50)), "p99_ms": float(np.percentile(a, 99)), "steps": int(a.size)}


def bench_volume(args, world, local):
    """Volume leg: one batched-volume scene (filtered 256^3 foliage medium +
    81,920-tri mesh), 1920x1080, depth 16, brick-grid DDA tracking."""
    import tempfile

    import torch
    from renderer2_b200 import raytracer as R
    from renderer2_b200 import render_scenes as RS
    c = VOLUME_CFG
    work = tempfile.mkdtemp(prefix="r2vol")
    desc, cam = RS.volume_scene(work, 0, grid=c["grid"], n_quads=c["n_quads"], ico_subdiv=c["ico_subdiv"],
                                width=c["width"], height=c["height"])
    prm = R.params(c["spp"], c["depth"], c["seed"], brick_grid=True)
    sc = RS.build_scene(desc)
    tuning = sc.autotune(cam, prm).as_dict()
    npix = cam.width * cam.height
    frame = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(args.warmup):
        sc.render_device(cam, prm, frame.data_ptr(), stream)
    torch.cuda.synchronize()
    _barrier(world)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    st = np.zeros(8)
    stats = []
    ev0.record()
    for _ in range(args.steps):
        # wave state (~1 GB at 1080p) and grid leaves exceed L2; no flush needed
        sc.render_device(cam, prm, frame.data_ptr(), stream, stats=st)
        stats.append(st.copy())
    ev1.record()
    torch.cuda.synchronize()
    _barrier(world)
    total_ms = _max_over_ranks(ev0.elapsed_time(ev1), world)
    paths = npix * prm.spp
    latency = step_latency([x[1] for x in stats])
    st = np.mean(np.array(stats), axis=0)
    seg, shadow = st[2], st[3]
    S = sc.wave_samples(cam, prm)
    roofline = media_roofline(st, S, prm.spp, prm.max_depth)
    ms_wave = roofline["kernel_ms_per_wave"]
    h2d = _input_bytes(desc) + sum(os.path.getsize(m[0] + e) for m in desc["media"] for e in (".nvdb", ".brickgrid"))
    e2e_ms = []
    for _ in range(1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s2 = RS.build_scene(desc)
        s2.render(cam, prm)
        s2.close()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = _max_over_ranks(float(np.median(e2e_ms)), world)
    sc.close()
    out = {"metric": "paths/s", "value": world * paths * args.steps / (total_ms / 1e3), "unit": "paths/s",
           "ms_per_step": total_ms / args.steps,
           "config": {"workload": f"batched volume scene 0: foliage {c['n_quads']} quads filtered to "
                                  f"{c['grid']}^3 (SGGX medium, brick-grid DDA) + {20 * 4 ** c['ico_subdiv']}-tri "
                                  f"mesh, {c['width']}x{c['height']}, {c['spp']} spp per step, depth {c['depth']}",
                      "paths_per_step": paths, "segments_per_step": seg, "shadow_rays_per_step": shadow,
                      "l2": "wave state larger than L2",
                      "tuning": tuning},
           "roofline": roofline, "latency": latency,
           "e2e": {"value": world * paths / (e2e_ms / 1e3), "unit": "paths/s", "h2d_bytes_per_step": int(h2d),
                   "d2h_bytes_per_step": int(npix * 12), "ms_per_step": e2e_ms},
           # per wave: camera, finish; per bounce: _media_launches
           "gpu_launches": (prm.spp // S) * (2 + _media_launches(tuning) * prm.max_depth) * args.steps}
    return out, (desc, cam, prm)


def bench_forest(args, world, local, cfg=None, autotune=True):
    """Forest leg: a many-instance scene as the reference's forest generator
    makes it (dart-throwing placement, screen-space LOD per tree; the trees
    nearest the camera stay meshes), medium instances sharing their files and
    walked through the instance BVH, 1920x1080, depth 16, brick-grid DDA.
    Also times the LOD selection of all trees (r2_select_lods) against the
    oracle's restatement on the host cores."""
    import tempfile

    import oracle_lib as O
    import torch
    from renderer2_b200 import forest as FO
    from renderer2_b200 import raytracer as R
    from renderer2_b200 import render_scenes as RS
    c = dict(FOREST_CFG, **(cfg or {}))
    work = tempfile.mkdtemp(prefix="r2forest")
    lib = RS.forest_library(work, n_quads=c["n_quads"], grid=c["grid"], lods=c["lods"])
    t0 = time.perf_counter()
    placed = FO.place_trees(lib["relevant_models"], lib["volume_descriptions"], c["attempts"], c["seed"], c["radius"])
    place_s = time.perf_counter() - t0
    pos, look, up, fov = RS.FOREST_CAMERA
    lcam = FO.lod_camera(pos, look, up, c["width"], c["height"], fov)
    table = FO.LodTable(lib["volume_descriptions"], sorted(lib["volume_descriptions"]))
    tp = np.array([p["Pos"] for p in placed])
    ts = np.array([p["Scaling"] for p in placed])
    tm = np.array([table.index[p["Model"]["Name"]] for p in placed], np.uint32)
    sel_ms = []
    for _ in range(5):
        t0 = time.perf_counter()
        choice = FO.select_lods(lcam, table, tp, ts, tm, c["min_lod"], c["covered_pixels"])
        sel_ms.append((time.perf_counter() - t0) * 1e3)
    t0 = time.perf_counter()
    n_cpu = min(len(placed), 20_000)
    ref = O.select_lods(lcam["native"], table.lods, table.first, table.count, tp[:n_cpu], ts[:n_cpu], tm[:n_cpu],
                        c["min_lod"], c["covered_pixels"])
    cpu_s = time.perf_counter() - t0
    assert np.array_equal(ref, choice[:n_cpu]), "LOD selection differs from the oracle"
    trees = RS.forest_trees(lib, c["attempts"], c["radius"], c["width"], c["height"], c["min_lod"],
                            c["covered_pixels"], placed=placed)
    desc = RS.forest_desc(lib, trees)
    t0 = time.perf_counter()
    sc = RS.build_scene(desc)
    build_ms = (time.perf_counter() - t0) * 1e3
    cam = R.camera(c["width"], c["height"], fov, pos, look, up)
    prm = R.params(c["spp"], c["depth"], c["seed"], brick_grid=True)
    tuning = sc.autotune(cam, prm).as_dict() if autotune else sc.get_tuning().as_dict()
    npix = cam.width * cam.height
    frame = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(args.warmup):
        sc.render_device(cam, prm, frame.data_ptr(), stream)
    torch.cuda.synchronize()
    _barrier(world)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    st = np.zeros(8)
    stats = []
    ev0.record()
    for _ in range(args.steps):
        # wave state (~1 GB at 1080p) exceeds L2; no flush needed
        sc.render_device(cam, prm, frame.data_ptr(), stream, stats=st)
        stats.append(st.copy())
    ev1.record()
    torch.cuda.synchronize()
    _barrier(world)
    total_ms = _max_over_ranks(ev0.elapsed_time(ev1), world)
    S = sc.wave_samples(cam, prm)
    bvh_nodes, bvh_height, _ = sc.bvh_info()
    sc.close()
    st = np.mean(np.array(stats), axis=0)
    roofline = media_roofline(st, S, prm.spp, prm.max_depth)
    latency = step_latency([x[1] for x in stats])
    paths = npix * prm.spp
    kinds = [t[0] for t in trees]
    lods = {}
    for t in trees:
        if t[0] == "Medium":
            lods[t[2]] = lods.get(t[2], 0) + 1
    return {"metric": "paths/s", "value": world * paths * args.steps / (total_ms / 1e3), "unit": "paths/s",
            "ms_per_step": total_ms / args.steps,
            "config": {"workload": f"forest: {kinds.count('Medium')} medium instances of {len(table.models)} tree "
                                   f"models x {c['lods']} LODs (finest {c['grid']} voxels tall) + "
                                   f"{kinds.count('Mesh')} mesh trees ({2 * c['n_quads']} tris each), disc radius "
                                   f"{c['radius']:g}, {c['width']}x{c['height']}, {c['spp']} spp per step, "
                                   f"depth {c['depth']}",
                       "trees": len(trees), "medium_instances": kinds.count("Medium"),
                       "mesh_trees": kinds.count("Mesh"), "lods": dict(sorted(lods.items())),
                       "paths_per_step": paths, "segments_per_step": st[2], "shadow_rays_per_step": st[3],
                       "kernel_ms_per_step": {"extend": st[4], "shade": st[5], "shadow": st[6], "accum": st[7]},
                       "bvh": {"two_level": kinds.count("Mesh") > 1, "inner_nodes": bvh_nodes,
                               "height": bvh_height},
                       "l2": "wave state larger than L2", "tuning": tuning},
            "roofline": roofline, "latency": latency,
            "lod_selection": {"trees": len(placed), "ms": float(np.median(sel_ms)),
                              "trees_per_s": len(placed) / (float(np.median(sel_ms)) / 1e3),
                              "timed": "r2_select_lods with host buffers (upload, kernel, download)",
                              "cpu_baseline": {"value": n_cpu / cpu_s, "unit": "trees/s", "cores": 1,
                                               "kind": "port", "sample": f"{n_cpu} trees"},
                              "placement_s": place_s, "placement_attempts": c["attempts"]},
            "scene_build_ms": build_ms,
            # per wave: camera, finish; per bounce: _media_launches
            "gpu_launches": (prm.spp // S) * (2 + _media_launches(tuning) * prm.max_depth) * args.steps}


def bench_volume_batch(args, world, local):
    """Batched volume leg: VOLUME_BATCH_CFG['scenes'] scenes (foliage grids of uneven size and
    occupancy filtered on the GPU, icosphere meshes of 82k or 328k triangles), 1920x1080, depth 16,
    brick-grid DDA, all rendered by one captured CUDA graph (a wave of every scene per replay);
    against the same frames rendered one scene after the other."""
    import shutil
    import tempfile

    import torch
    from renderer2_b200 import raytracer as R
    from renderer2_b200 import render_scenes as RS
    c = VOLUME_BATCH_CFG
    work = tempfile.mkdtemp(prefix="r2vb")
    descs, cams, prms = [], [], []
    for i in range(c["scenes"]):
        d, cam = RS.volume_scene(work, 100 + i, grid=c["grids"][i % len(c["grids"])],
                                 n_quads=c["quads"][(i // 2) % len(c["quads"])], ico_subdiv=c["ico"][i % 2],
                                 width=c["width"], height=c["height"])
        descs.append(d)
        cams.append(cam)
        prms.append(R.params(c["spp"], c["depth"], i, brick_grid=True))
    scs = [RS.build_scene(d) for d in descs]
    tuned = scs[0].autotune(cams[0], prms[0])  # one scene's choice applies to all
    for sc in scs[1:]:
        sc.set_tuning(tuned)
    npix = [cm.width * cm.height for cm in cams]
    frames = [torch.empty(n * 3, dtype=torch.float32, device="cuda") for n in npix]
    stream = torch.cuda.current_stream().cuda_stream
    # the batch's own tracker occupancy (its graph runs every scene's wave at once, so fewer tracker
    # blocks per branch can pay where one scene alone wants them all): set-up, untimed
    best = None
    for blocks in (tuned.track_blocks, 4, 3):
        t = R.tuning(*tuned.as_tuple()[:5], blocks)
        for sc in scs:
            sc.set_tuning(t)
        b = R.RenderBatch(scs, cams, prms, [f.data_ptr() for f in frames])
        b.run(stream, timing=False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.run(stream, timing=False)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        b.close()
        if best is None or dt < best[0] * 0.98:
            best = (dt, t)
    batch_tuning = best[1]
    for sc in scs:
        sc.set_tuning(batch_tuning)
    batch = R.RenderBatch(scs, cams, prms, [f.data_ptr() for f in frames])
    for sc in scs:  # one scene at a time keeps the scene's own tuning
        sc.set_tuning(tuned)
    for _ in range(args.warmup):
        batch.run(stream, timing=False)
        for sc, cm, p, f in zip(scs, cams, prms, frames):
            sc.render_device(cm, p, f.data_ptr(), stream)
    torch.cuda.synchronize()
    _barrier(world)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        # 16 scenes' wave state (~1 GB each) and media exceed L2; no flush needed
        evs[k][0].record()
        batch.run(stream, timing=False)
        evs[k][1].record()
    ev[1].record()
    sst = [np.zeros(8) for _ in scs]
    for _ in range(args.steps):
        for k, (sc, cm, p, f) in enumerate(zip(scs, cams, prms, frames)):
            st = np.zeros(8)
            sc.render_device(cm, p, f.data_ptr(), stream, stats=st)
            sst[k] += st / args.steps
    ev[2].record()
    torch.cuda.synchronize()
    _barrier(world)
    ms_batch = _max_over_ranks(ev[0].elapsed_time(ev[1]), world)
    ms_seq = _max_over_ranks(ev[1].elapsed_time(ev[2]), world)
    latency = step_latency([a.elapsed_time(b) for a, b in evs])
    # roofline of the dominant phase, scene by scene (statistics of the one-at-a-time frames)
    rfs = [media_roofline(st, sc.wave_samples(cm, p), p.spp, p.max_depth) for st, sc, cm, p in zip(sst, scs, cams, prms)]
    w = np.array([sum(r["kernel_ms_per_wave"].values()) for r in rfs])
    roofline = dict(rfs[0])
    roofline["frac"] = float(np.sum(w * np.array([r["frac"] for r in rfs])) / np.sum(w))
    roofline["achieved"] = roofline["frac"] * roofline["peak"]
    roofline["note"] = ("time-weighted mean over the 16 scenes of each scene's dominant phase, from its frame rendered "
                        "alone; " + rfs[0]["note"])
    roofline["per_scene_frac"] = [round(r["frac"], 5) for r in rfs]
    paths = sum(npix) * c["spp"]
    # end to end: upload every scene (media read from their files), one batch, frames back to the host
    h2d = sum(_input_bytes(d) + sum(os.path.getsize(m[0] + e) for m in d["media"] for e in (".nvdb", ".brickgrid"))
              for d in descs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s2 = [RS.build_scene(d) for d in descs]
    b2 = R.RenderBatch(s2, cams, prms, [f.data_ptr() for f in frames])
    b2.run(stream, timing=False)
    host = [f.cpu().numpy() for f in frames]
    e2e_ms = _max_over_ranks((time.perf_counter() - t0) * 1e3, world)
    b2.close()
    for s in s2:
        s.close()
    batch.close()
    for s in scs:
        s.close()
    del host
    shutil.rmtree(work, ignore_errors=True)
    return {"metric": "paths/s", "value": world * paths * args.steps / (ms_batch / 1e3), "unit": "paths/s",
            "ms_per_step": ms_batch / args.steps,
            "config": {"workload": f"{c['scenes']} batched volume scenes: foliage grids {sorted(set(c['grids']))}^3 of "
                                   f"{c['quads']} quads (SGGX media, brick-grid DDA) + icosphere meshes "
                                   f"(81,920 / 327,680 tris), {c['width']}x{c['height']}, {c['spp']} spp per step, "
                                   f"depth {c['depth']}, one captured graph per sample",
                       "paths_per_step": paths, "l2": "wave state larger than L2",
                       "tuning": batch_tuning.as_dict(), "scene_tuning": tuned.as_dict()},
            "one_scene_at_a_time": {"value": world * paths * args.steps / (ms_seq / 1e3),
                                    "ms_per_step": ms_seq / args.steps},
            "speedup_vs_one_at_a_time": ms_seq / ms_batch,
            "roofline": roofline, "latency": latency,
            "frames_256spp_ms": ms_batch / args.steps / c["spp"] * c["frame_spp"],
            "frames_256spp_note": "the 16 frames at the configuration's 256 spp: the graph replays one sample of every "
                                  "scene per replay, so a full frame set is 256 replays; time per replay measured "
                                  f"over {args.steps} steps of {c['spp']} replays",
            "e2e": {"value": world * paths / (e2e_ms / 1e3), "unit": "paths/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(sum(npix) * 12), "ms_per_step": e2e_ms},
            "gpu_launches": c["spp"] * c["scenes"] * (3 + _media_launches(tuned.as_dict()) * c["depth"]) * args.steps}


def serving_jobs(c=SERVE_CFG, seed=11):
    """A serving mix: c['jobs'] jobs, Poisson arrivals at c['rate'] per second; 70% renders (sizes c['sizes'],
    spp log-uniform in c['spp'], depth 8, on the small icosphere and the icosphere-grid scenes), 30% filter
    jobs (grids c['grids'] over foliage of c['quads'] leaf quads, 64 spv, 10 iterations).  SERVE_CFG is the
    mix scaled to a bench step (256^2 .. 1280x720, spp 4 .. 64, 64^3 .. 192^3, 20k .. 200k triangles)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    sizes = list(c["sizes"])
    lo, hi = c["spp"]
    for k in range(c["jobs"]):
        t += float(rng.exponential(1.0 / c["rate"]))
        if rng.uniform() < 0.7:
            w, h = sizes[int(rng.integers(len(sizes)))]
            spp = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
            jobs.append(("render", t, int(rng.integers(2)), w, h, spp, int(rng.integers(1 << 30))))
        else:
            jobs.append(("filter", t, int(rng.integers(len(c["quads"]))), int(rng.choice(list(c["grids"]))),
                         int(rng.integers(1 << 30))))
    return jobs


def bench_serving(args, c=SERVE_CFG):
    """Served (request loop, c['slots'] slots) against one job at a time on the same GPU."""
    import threading as th

    import torch
    from renderer2_b200 import filter as F
    from renderer2_b200 import raytracer as R
    from renderer2_b200 import render_scenes as RS
    from renderer2_b200 import scenes
    from renderer2_b200 import serving as S
    d1, _ = RS.icosphere_scene()
    d2, _ = RS.icosphere_grid_scene()
    rscenes = [RS.build_scene(d1), RS.build_scene(d2)]
    cams = [((0, 0, 3), (0, 0, 0)), ((0, 0, 24), (0, 0, 0))]
    fmat = F.material(diffuse=(0.1, 0.6, 0.1), specular=(0.04, 0.04, 0.04), alpha=0.5, ior=1.5)
    meshes = [scenes.foliage(n, 10, 0.7, 20 + i) for i, n in enumerate(c["quads"])]
    fscenes = [F.FilterScene(m, fmat) for m in meshes]
    jobs = serving_jobs(c)

    def spec(j):
        if j[0] == "render":
            _, _, si, w, h, spp, seed = j
            pos, at = cams[si]
            return rscenes[si], R.camera(w, h, 45.0, pos, at, (0, 1, 0)), R.params(spp, 8, seed)
        _, _, fi, n, seed = j
        return fscenes[fi], fscenes[fi].grid(scenes.voxel_size_for(meshes[fi], n)), \
            F.params(samples_per_voxel=64, iterations=10, seed=seed)

    specs = [spec(j) for j in jobs]
    work = [(s[1].width * s[1].height * s[2].spp, 0) if j[0] == "render" else
            (0, int(np.prod(np.array(s[1].num_voxels[:], np.int64)))) for j, s in zip(jobs, specs)]
    paths, voxels = sum(w[0] for w in work), sum(w[1] for w in work)
    arrivals = np.array([j[1] for j in jobs])

    def run_alone(k):
        s = specs[k]
        if jobs[k][0] == "render":
            s[0].render(s[1], s[2])
        else:
            nvox = work[k][1]
            out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
            s[0].run(s[1], s[2], out.data_ptr())
            out.cpu()
        torch.cuda.synchronize()

    for k in range(min(4, len(jobs))):  # warm-up (BVH and graph code paths, allocations)
        run_alone(k)

    def one_at_a_time(arr):
        """FIFO on one queue, each job alone on the GPU; completion times from the first arrival."""
        t0 = time.perf_counter()
        done = []
        for k in range(len(jobs)):
            now = time.perf_counter() - t0
            if now < arr[k]:
                time.sleep(arr[k] - now)
            run_alone(k)
            done.append(time.perf_counter() - t0)
        return done[-1] - arr[0], np.array(done) - arr

    srv = S.Server(slots=c["slots"], hbm_budget=c["budget"])
    # warm-up like the one-at-a-time path: the largest job of each kind, submitted once per slot at the same
    # time so that each slot takes one and sizes its buffers (grow-only) before the timed runs
    big = sorted(range(len(jobs)), key=lambda k: -(work[k][0] + 64 * work[k][1]))
    warm = [big[0]] + [k for k in big if jobs[k][0] != jobs[big[0]][0]][:1]
    for k in warm:
        hs = [srv.submit_render(*specs[k]) if jobs[k][0] == "render" else srv.submit_filter(*specs[k])
              for _ in range(c["slots"])]
        for h in hs:
            srv.wait(h, 600.0)

    def served(arr):
        """Submitted at the arrival times from another thread, served by the request loop."""
        handles = [None] * len(jobs)
        t0 = time.perf_counter()

        def submitter():
            for k in range(len(jobs)):
                now = time.perf_counter() - t0
                if now < arr[k]:
                    time.sleep(arr[k] - now)
                s = specs[k]
                handles[k] = srv.submit_render(*s) if jobs[k][0] == "render" else srv.submit_filter(*s)

        th_sub = th.Thread(target=submitter)
        th_sub.start()
        th_sub.join()
        done = np.zeros(len(jobs))
        for k in range(len(jobs)):
            srv.wait(handles[k], 600.0)
            done[k] = handles[k].times[2] - handles[k].times[0] + arr[k]
        return done.max() - arr[0], done - arr

    descs = [d1, d2]

    def plain(k):
        """A job as a process that renders one frame does it: build the scene (upload, BVH), run, download."""
        j = jobs[k]
        if j[0] == "render":
            sc = RS.build_scene(descs[j[2]])
            sc.render(specs[k][1], specs[k][2])
            sc.close()
        else:
            fs = F.FilterScene(meshes[j[2]], fmat)
            out = torch.empty(work[k][1] * 32, dtype=torch.uint8, device="cuda")
            fs.run(fs.grid(scenes.voxel_size_for(meshes[j[2]], j[3])), specs[k][2], out.data_ptr())
            out.cpu()
            fs.close()
        torch.cuda.synchronize()

    # Host-side timing (Python submission, sleeps to the arrival times) varies from run to run on a
    # shared host: each of the four measurements is taken three times, interleaved, and the run with the
    # median makespan is reported; the plain path (each job building its scene) the faster of two runs.
    burst = np.zeros(len(jobs))  # every job waiting at once: the throughput each path sustains
    reps = {"alone": [], "served": [], "alone_burst": [], "served_burst": []}
    for _ in range(3):
        reps["alone"].append(one_at_a_time(arrivals))
        reps["served"].append(served(arrivals))
        reps["alone_burst"].append(one_at_a_time(burst))
        reps["served_burst"].append(served(burst))

    def median_run(runs):
        return sorted(runs, key=lambda r: r[0])[len(runs) // 2]

    span_alone, lat_alone = median_run(reps["alone"])
    span_srv, lat_srv = median_run(reps["served"])
    span_alone_b, _ = median_run(reps["alone_burst"])
    span_srv_b, lat_srv_b = median_run(reps["served_burst"])
    plain(0)
    spans_plain = []
    for _ in range(2):
        t0 = time.perf_counter()
        for k in range(len(jobs)):
            plain(k)
        spans_plain.append(time.perf_counter() - t0)
    span_plain_b = min(spans_plain)
    srv.close()
    for sc in rscenes:
        sc.close()
    for fs in fscenes:
        fs.close()

    def pct(a, q):
        return float(np.percentile(a, q))

    return {"metric": "served paths/s & filtered voxels/s", "unit": "paths/s, voxels/s",
            "config": {"workload": f"{len(jobs)} jobs, Poisson arrivals at {c['rate']}/s: 70% renders "
                                   f"({c['sizes'][0][0]}x{c['sizes'][0][1]}..{c['sizes'][-1][0]}x{c['sizes'][-1][1]}, "
                                   f"spp log-uniform {c['spp'][0]}..{c['spp'][1]}, depth 8, icosphere / icosphere-grid "
                                   f"scenes), 30% filters ({c['grids'][0]}^3..{c['grids'][-1]}^3, foliage "
                                   f"{c['quads'][0]}..{c['quads'][-1]} quads, 64 spv, 10 iterations)",
                       "slots": c["slots"], "hbm_budget_bytes": c["budget"], "paths": paths, "voxels": voxels},
            "served": {"paths_per_s": paths / span_srv, "voxels_per_s": voxels / span_srv, "makespan_s": span_srv,
                       "p50_latency_s": pct(lat_srv, 50), "p99_latency_s": pct(lat_srv, 99)},
            "one_at_a_time": {"paths_per_s": paths / span_alone, "voxels_per_s": voxels / span_alone,
                              "makespan_s": span_alone, "p50_latency_s": pct(lat_alone, 50),
                              "p99_latency_s": pct(lat_alone, 99)},
            "speedup_makespan": span_alone / span_srv,
            "makespans_s": {k: [round(r[0], 4) for r in v] for k, v in reps.items()} | {"plain_burst": spans_plain},
            "burst": {"workload": f"the same {len(jobs)} jobs all submitted at once",
                      "served": {"paths_per_s": paths / span_srv_b, "voxels_per_s": voxels / span_srv_b,
                                 "makespan_s": span_srv_b, "p50_latency_s": pct(lat_srv_b, 50),
                                 "p99_latency_s": pct(lat_srv_b, 99)},
                      "one_at_a_time": {"paths_per_s": paths / span_alone_b, "voxels_per_s": voxels / span_alone_b,
                                        "makespan_s": span_alone_b},
                      "speedup_makespan": span_alone_b / span_srv_b,
                      "plain_per_job_scene_build": {
                          "paths_per_s": paths / span_plain_b, "voxels_per_s": voxels / span_plain_b,
                          "makespan_s": span_plain_b,
                          "note": "each job builds its scene (upload, BVH), runs and downloads, one after the "
                                  "other; the faster of two runs"},
                      "speedup_vs_plain": span_plain_b / span_srv_b}}


def run_native(args):
    import torch
    world, rank, local = _dist_setup()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    import renderer2_b200  # noqa: F401  (loads the native library)

    if args.skip_render:
        f = bench_filter(args, world, local)
        if rank == 0:
            mesh, mat, prm, vs = f.pop("_mesh")
            f.pop("_gpu_slab")
            f.update({"n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)"})
            if world == 1:
                f["cpu_baseline"] = cpu_filter_sample(mesh, mat, prm, vs, budget_s=args.cpu_budget)
            print(json.dumps(f), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    r = bench_render(args, world, local)
    small = bench_small(args, world, local) if not args.skip_small else None
    f = bench_filter(args, world, local) if not args.skip_filter else None
    f512 = None
    if f is not None and not args.skip_512:
        mesh1m, mat1m = f["_mesh"][0], f["_mesh"][1]
        f512 = bench_filter(args, world, local, grid=512, steps=1, warmup=1, e2e_run=False, mesh_mat=(mesh1m, mat1m))
    vol = bench_volume(args, world, local) if not args.skip_volume else None
    vbatch = bench_volume_batch(args, world, local) if not args.skip_volume else None
    forest = bench_forest(args, world, local) if not args.skip_volume else None
    serve = bench_serving(args) if (not args.skip_serving and world == 1) else None
    if rank == 0:
        cpu = cpu_render_baseline(r["desc"], r["cam"], r["prm"], budget_s=args.cpu_budget) if world == 1 else None
        line = {"metric": "paths/s", "value": r["value"], "unit": "paths/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["total_ms"] / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
                "config": headline_config(world),
                "workload_stats": {"segments_per_step": r["segments_per_frame"],
                                   "shadow_rays_per_step": r["shadow_rays_per_frame"],
                                   "bvh_build_ms_per_step": r["bvh_build_ms"], "render_ms_per_step": r["render_ms"],
                                   "bvh": r["bvh"], "tuning": r["tuning"]},
                "roofline": r["roofline"], "cpu_baseline": cpu, "e2e": r["e2e"], "gpu_launches": r["launches"],
                "latency": r["latency"], "clocks": r["clocks"]}
        if small is not None:
            line["small"] = small
            line["gpu_launches"] += small["gpu_launches"]
        for key, leg in (("filter", f), ("filter_512", f512)):
            if leg is None:
                continue
            mesh, mat, prm, vs = leg.pop("_mesh")
            (v0, v1), (gw, gh) = leg.pop("_gpu_slab")
            if world == 1:
                keep = {}
                budget = args.cpu_budget if key == "filter" else max(5.0, args.cpu_budget / 2)
                leg["cpu_baseline"] = cpu_filter_sample(mesh, mat, prm, vs, budget_s=budget, keep=keep)
                if keep.get("v0") == v0 and keep.get("v1") == v1:
                    leg["accuracy"] = filter_accuracy(gw, gh, keep["wide"])
                    leg["accuracy"]["sample"] = "the central z-slice, FP32 records and FP16 payload vs the FP64 oracle"
            line[key] = leg
            line["gpu_launches"] += leg["gpu_launches"]
        if vol is not None:
            v, (vdesc, vcam, vprm) = vol
            if world == 1:
                v["cpu_baseline"] = cpu_render_sample(vdesc, vcam, vprm, budget_s=max(5.0, args.cpu_budget / 2))
            line["volume"] = v
            line["gpu_launches"] += v["gpu_launches"]
        if vbatch is not None:
            line["volume_batch"] = vbatch
            line["gpu_launches"] += vbatch["gpu_launches"]
        if forest is not None:
            line["forest"] = forest
            line["gpu_launches"] += forest["gpu_launches"]
        if serve is not None:
            line["serving"] = serve
        line["legs"] = legs_summary(line)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _short(x, nd=4):
    return None if x is None else float(f"{x:.{nd}g}")


def legs_summary(line: dict) -> dict:
    """One compact entry per leg (value, e2e, roofline fraction, latency), kept at the end of the line."""
    out = {}

    def leg(name, d, value_key="value"):
        if not d:
            return
        e = {"value": _short(d.get(value_key)), "unit": d.get("unit")}
        if isinstance(d.get("e2e"), dict):
            e["e2e"] = _short(d["e2e"].get("value"))
        rf = d.get("roofline")
        if isinstance(rf, dict):
            e["hbm_frac"] = _short(rf.get("frac"), 3)
            if isinstance(rf.get("fp32"), dict):
                e["fp32_frac"] = _short(rf["fp32"].get("frac"), 3)
        for k in ("paths_per_s", "p50_latency_s", "p99_latency_s", "speedup_vs_one_at_a_time"):
            if k in d:
                e[k] = _short(d[k], 4)
        if isinstance(d.get("latency"), dict):
            e["p99_step_ms"] = _short(d["latency"]["p99_ms"], 4)
        if isinstance(rf, dict) and "filter" in rf and "render" in rf:
            e["hbm_frac"] = {"filter": _short(rf["filter"]["frac"], 3), "render": _short(rf["render"]["frac"], 3)}
        acc = d.get("accuracy")
        if isinstance(acc, dict):
            fa = acc.get("filter", acc)
            if "fp16" in fa:
                e["fp16_vs_fp64"] = _short(max(fa["fp16"]["density"], fa["fp16"]["S"]), 3)
                e["fp32_vs_fp64"] = _short(max(fa["fp32"]["density"], fa["fp32"]["S"]), 3)
        out[name] = e

    leg("headline", line)
    for k in ("small", "filter", "filter_512", "volume", "volume_batch", "forest"):
        leg(k, line.get(k))
    sv = line.get("serving")
    if sv:
        out["serving"] = {"paths_per_s": _short(sv["served"]["paths_per_s"]),
                          "voxels_per_s": _short(sv["served"]["voxels_per_s"]),
                          "p50_latency_s": _short(sv["served"]["p50_latency_s"], 3),
                          "p99_latency_s": _short(sv["served"]["p99_latency_s"], 3),
                          "speedup_makespan": _short(sv.get("speedup_makespan"), 3),
                          "burst_speedup_vs_one_at_a_time": _short(sv["burst"].get("speedup_makespan"), 3),
                          "burst_speedup_vs_plain": _short(sv["burst"].get("speedup_vs_plain"), 3)}
        if isinstance(sv.get("roofline"), dict):
            out["serving"]["hbm_frac"] = _short(sv["roofline"].get("frac"), 3)
    return out


def run_reference(args):
    world, rank, _ = _dist_setup()
    if rank != 0:
        return
    desc, cam, prm = render_workload()
    for _ in range(args.warmup):
        cpu_render_baseline(desc, cam, prm, budget_s=1.0)
    vals = [cpu_render_baseline(desc, cam, prm, budget_s=args.cpu_budget / max(1, args.steps))
            for _ in range(args.steps)]
    v = float(np.median([x["value"] for x in vals]))
    cpu = dict(vals[-1])
    cpu["value"] = v
    # beside it: the oracle port at the configuration's depth (the reference integrator's bounce cap is its own)
    port = cpu_render_sample(desc, cam, prm, budget_s=max(3.0, args.cpu_budget / 2)) if cpu["kind"] != "port" else None
    line = {"impl": "reference", "metric": "paths/s", "value": v, "unit": "paths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * float(np.mean([x["seconds"] for x in vals])),  # a bounded sample per step
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
            "config": headline_config(world),
            "cpu_baseline": cpu,
            "e2e": {"value": v, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "oracle_port": port}
    if not args.skip_filter:
        mesh, mat, fprm, vs = filter_workload()
        budget = max(5.0, args.cpu_budget / 2)
        fc = ref_code_filter_sample(mesh, mat, fprm, vs, budget_s=budget)
        fport = cpu_filter_sample(mesh, mat, fprm, vs, budget_s=budget)
        if fc is None:
            fc, fport = fport, None
        line["filter"] = {"metric": "filtered voxels/s", "value": fc["value"], "unit": "voxels/s", "cpu_baseline": fc,
                          "oracle_port": fport}
    # the CPU arm runs the oracle (and the host-compiled reference) alone: the GPU library must not be in this process
    with open("/proc/self/maps") as fh:
        assert "librenderer2" not in fh.read(), "the reference arm loaded the GPU library"
    line["native_libraries"] = "oracle only"
    print(json.dumps(line), flush=True)


def run_case(args):
    """Small single-GPU cases for kernel profiling (a few hundred MB on the device)."""
    import torch
    torch.cuda.set_device(0)
    if args.case == "render-small":
        from renderer2_b200 import render_scenes as RS
        from renderer2_b200 import raytracer as R
        desc, _ = RS.icosphere_grid_scene()
        cam = R.camera(256, 256, 45.0, (0, 0, 24), (0, 0, 0), (0, 1, 0))
        sc = RS.build_scene(desc)
        frame = torch.empty(256 * 256 * 3, dtype=torch.float32, device="cuda")
        st = sc.render_device(cam, R.params(2, 8, 0), frame.data_ptr())
        torch.cuda.synchronize()
        sc.close()
        print(json.dumps({"case": args.case, "paths": st[0], "ms": st[1]}))
    elif args.case == "render-wave":
        # one wave of the headline frame: --case-spp samples of every pixel in one wave
        desc, cam, prm = render_workload()
        from renderer2_b200 import render_scenes as RS
        from renderer2_b200 import raytracer as R
        sc = RS.build_scene(desc)
        frame = torch.empty(cam.width * cam.height * 3, dtype=torch.float32, device="cuda")
        n = args.case_spp
        sc.set_tuning(R.tuning(wave_paths=cam.width * cam.height * n))
        st = sc.render_device(cam, R.params(n, prm.max_depth, 0), frame.data_ptr())
        torch.cuda.synchronize()
        sc.close()
        print(json.dumps({"case": args.case, "paths": st[0], "segments": st[2], "shadow_rays": st[3], "ms": st[1],
                          "ms_per_wave": {"extend": st[4], "shade": st[5], "shadow": st[6], "accum": st[7]}}))
    elif args.case in ("filter-small", "filter-mid"):
        from renderer2_b200 import filter as F
        from renderer2_b200 import scenes
        # small: 100k leaf quads at 64^3 (dense voxels); mid: 62.5k quads at 128^3, the 256^3 filter's
        # triangles per voxel at an eighth of its size
        nq, n = (100_000, 64) if args.case == "filter-small" else (62_500, 128)
        mesh = scenes.foliage(nq, 20, 0.7, 4)
        mat = F.material(diffuse=(0.1, 0.6, 0.1), specular=(0.04, 0.04, 0.04), alpha=0.5, ior=1.5)
        sc = F.FilterScene(mesh, mat)
        g = sc.grid(scenes.voxel_size_for(mesh, n))
        nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
        out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
        st = np.zeros(3)
        sc.run(g, F.params(samples_per_voxel=256, iterations=20), out.data_ptr(), stats=st)
        torch.cuda.synchronize()
        sc.close()
        print(json.dumps({"case": args.case, "voxels": st[0], "candidates": st[1], "ms": st[2]}))
    elif args.case == "serving":
        import renderer2_b200  # noqa: F401
        print(json.dumps(bench_serving(args)))
    elif args.case == "serving-stated":  # the serving configuration's own mix and sizes
        import renderer2_b200  # noqa: F401
        print(json.dumps(bench_serving(args, SERVE_CFG_STATED)))
    elif args.case == "volume-batch":
        import renderer2_b200  # noqa: F401
        args.steps, args.warmup = 1, 1
        print(json.dumps(bench_volume_batch(args, 1, 0)))
    elif args.case == "forest":
        args.steps, args.warmup = 1, 1
        print(json.dumps(bench_forest(args, 1, 0)))
    elif args.case == "forest-small":  # a quarter of the pixels, 1 spp, default tuning: one wave per step
        args.steps, args.warmup = 1, 1
        print(json.dumps(bench_forest(args, 1, 0, dict(width=960, height=540, spp=1), autotune=False)))
    elif args.case in ("volume-small", "volume-mid"):
        import tempfile

        from renderer2_b200 import raytracer as R
        from renderer2_b200 import render_scenes as RS
        if args.case == "volume-small":
            desc, cam = RS.volume_scene(tempfile.mkdtemp(prefix="r2vol"), 0, grid=128, n_quads=50_000, ico_subdiv=4,
                                        width=480, height=270)
        else:  # the bench scene at a quarter of the pixels, one wave
            desc, cam = RS.volume_scene(tempfile.mkdtemp(prefix="r2vol"), 0, width=960, height=540)
        sc = RS.build_scene(desc)
        frame = torch.empty(cam.width * cam.height * 3, dtype=torch.float32, device="cuda")
        spp = 2 if args.case == "volume-small" else 1
        st = sc.render_device(cam, R.params(spp, 16, 0, brick_grid=True), frame.data_ptr())
        torch.cuda.synchronize()
        sc.close()
        print(json.dumps({"case": args.case, "paths": st[0], "ms": st[1], "extend_ms": st[4], "shade_ms": st[5],
                          "shadow_ms": st[6]}))
    else:
        raise SystemExit(f"unknown case {args.case}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--skip-filter", action="store_true")
    ap.add_argument("--skip-volume", action="store_true")
    ap.add_argument("--skip-serving", action="store_true")
    ap.add_argument("--skip-render", action="store_true", help="run only the filter leg")
    ap.add_argument("--skip-small", action="store_true", help="skip the small configuration's leg")
    ap.add_argument("--skip-512", action="store_true", help="skip the 512^3 filter leg")
    ap.add_argument("--case", default=None,
                    help="profiling case: render-wave | filter-small | filter-mid | volume-small | volume-mid | volume-batch | forest | "
                         "forest-small | serving | serving-stated")
    ap.add_argument("--case-spp", type=int, default=1, help="render-wave: samples per pixel, all in one wave")
    args = ap.parse_args()
    if args.case:
        run_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_native(args)


if __name__ == "__main__":
    main()
