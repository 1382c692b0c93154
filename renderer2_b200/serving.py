"""Python view of the request loop (r2_server_*): render and filter jobs
admitted into device slots under an HBM budget, overlapping on the GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class Job:
    def __init__(self, jid: int, out: np.ndarray, kind: str):
        self.id = jid
        self.out = out
        self.kind = kind
        self.times = None  # submit, start, end (seconds on the server clock)


class Server:
    def __init__(self, slots: int = 4, hbm_budget: int = 64 << 30):
        h = C.c_void_p()
        N.check(N.lib.r2_server_create(int(slots), int(hbm_budget), C.byref(h)))
        self.handle = h
        self._keep = {}

    def close(self):
        if self.handle:
            N.check(N.lib.r2_server_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def render_bytes(scene, camera, params) -> int:
        """Device bytes a render job is admitted with (r2_server_render_bytes)."""
        b = C.c_uint64()
        N.check(N.lib.r2_server_render_bytes(scene.handle, C.byref(camera), C.byref(params), C.byref(b)))
        return b.value

    def submit_render(self, scene, camera, params) -> Job:
        out = np.zeros((camera.height, camera.width, 3), np.float32)
        jid = C.c_uint64()
        N.check(N.lib.r2_server_submit_render(self.handle, scene.handle, C.byref(camera), C.byref(params), N.ptr(out),
                                              C.byref(jid)))
        job = Job(jid.value, out, "render")
        self._keep[job.id] = (scene, camera, params)
        return job

    def submit_filter(self, fscene, grid, params, lod: int = 0) -> Job:
        n = int(np.prod(np.array(grid.num_voxels[:], np.int64)))
        out = np.zeros(n, N.VOXEL_DTYPE)
        jid = C.c_uint64()
        N.check(N.lib.r2_server_submit_filter(self.handle, fscene.handle, C.byref(grid), C.byref(params), int(lod),
                                              N.ptr(out), C.byref(jid)))
        job = Job(jid.value, out, "filter")
        self._keep[job.id] = (fscene, grid, params)
        return job

    def wait(self, job: Job, timeout: float = -1.0) -> bool:
        """True when the job finished (its array is filled); False on timeout."""
        t = np.zeros(3)
        st = N.lib.r2_server_wait(self.handle, job.id, float(timeout), N.ptr(t))
        if st == 10:  # R2_ERR_PENDING
            return False
        self._keep.pop(job.id, None)
        N.check(st)
        job.times = t.copy()
        return True

    def stats(self):
        s = np.zeros(5)
        N.check(N.lib.r2_server_stats(self.handle, N.ptr(s)))
        return {"done": s[0], "queued": s[1], "running": s[2], "bytes_admitted": s[3], "seconds": s[4]}
