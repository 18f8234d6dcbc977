"""Device voxelization (vf_inside_points / vf_inside_grid) against the
reference's own parity ray cast: bit-identical masks for random points, voxel
centers and grid nodes of three closed meshes (box, torus with a hole, rotated
box), plus the oracle on a larger random mesh."""

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["box", "torus", "tilted"])
def test_inside_matches_reference(gpu, name):
    from voxelsim_fea_b200 import inside
    g = golden("inside_cases.npz")
    dims, origin, vsize = tuple(int(v) for v in g["dims"]), g["origin"], float(g["vsize"])
    v, f = g[f"{name}_verts"], g[f"{name}_faces"]
    np.testing.assert_array_equal(inside.inside_mask(v, f, g[f"{name}_points"]), g[f"{name}_in_points"])
    np.testing.assert_array_equal(inside.inside_mask(v, f, g["centers"]), g[f"{name}_in_centers"])
    np.testing.assert_array_equal(inside.inside_grid(v, f, dims, origin, vsize, "centers"), g[f"{name}_in_centers"])
    np.testing.assert_array_equal(inside.inside_grid(v, f, dims, origin, vsize, "nodes"), g[f"{name}_in_nodes"])


def test_inside_matches_oracle_on_many_triangles(gpu):
    from oracle import voxelize
    from voxelsim_fea_b200 import inside
    sys_path_golden = golden("inside_cases.npz")
    v, f = sys_path_golden["torus_verts"], sys_path_golden["torus_faces"]
    # refine: many small triangles (the reference's numpy path at any size)
    rng = np.random.default_rng(9)
    pts = rng.uniform(-0.1, 1.1, size=(20000, 3))
    np.testing.assert_array_equal(inside.inside_mask(v, f, pts), voxelize.inside_mask(v, f, pts))
    assert inside.inside_mask(v, f, np.zeros((0, 3))).size == 0
    assert not inside.inside_mask(np.zeros((0, 3)), np.zeros((0, 3), dtype=np.int64), pts).any()
    with pytest.raises(ValueError):
        inside.inside_mask(v, np.array([[0, 1, len(v)]]), pts)   # face index out of range
