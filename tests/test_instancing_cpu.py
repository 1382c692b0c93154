"""Two-level scenes in the oracle: instances of one mesh asset (model-space
BVH, rays taken to object space) against the same meshes flattened into
world space.  The two differ only by rounding in the hit computations, so
their frames agree in the mean and in nearly every pixel."""
import numpy as np

import oracle_lib as O
from renderer2_b200 import render_scenes as RS


def test_oracle_instances_match_flattened_meshes():
    desc, cam = RS.instanced_scene(3, 32, 32)
    assert RS.mesh_groups(desc) == [list(range(9))]
    a = O.render(desc, cam, 16, 6, 5, instancing=True)
    b = O.render(desc, cam, 16, 6, 5, instancing=False)
    rel = (np.abs(a - b) / np.maximum(1.0, np.abs(b))).max(axis=1)
    print(f"instanced vs flattened: {(rel <= 1e-3).mean():.4f} of pixels within 1e-3, "
          f"means {a.mean(0)} / {b.mean(0)}")
    assert (rel <= 1e-3).mean() >= 0.9
    assert np.abs(a.mean(0) - b.mean(0)).max() <= 0.02 * np.abs(b.mean(0)).max()
    # the instances are seen: without them the frame changes
    bare = dict(desc, meshes=desc["meshes"][9:])
    c = O.render(bare, cam, 4, 6, 5)
    assert np.abs(c.mean(0) - b.mean(0)).max() > 0.02 * np.abs(b.mean(0)).max()
