"""Host model builder semantics, restating the reference's own unit tests for
the DOF system as behavioural specs:
modules/litho-surface/tests/test_dof_system.cpp, test_vertex_freedom.cpp,
modules/litho-model/tests/test_global_dofs.cpp, test_no_gap.cpp."""
import numpy as np
import pytest

from lithoinv3d_b200 import FIXED, XYZ_FREE, Z_ONLY, LithoError, Model
from lithoinv3d_b200.api import ALONG_VECTOR, X_ONLY, XY_FREE, XZ_FREE, Y_ONLY, YZ_FREE


def one_vertex_model(freedom, pos=(10.0, 20.0, 30.0)):
    m = Model()
    m.add_group(0, 1.0)
    m.set_group_mesh(0, np.array([pos]), np.array([[0, 0, 0]]), [freedom])
    return m


@pytest.mark.parametrize("freedom,count", [(FIXED, 0), (Z_ONLY, 1), (X_ONLY, 1), (Y_ONLY, 1), (ALONG_VECTOR, 1),
                                           (XY_FREE, 2), (XZ_FREE, 2), (YZ_FREE, 2), (XYZ_FREE, 3)])
def test_dof_counting(freedom, count):
    # test_vertex_freedom.cpp:7-67
    assert one_vertex_model(freedom).n_dofs == count


def test_apply_respects_freedom_and_scale():
    # test_dof_system.cpp:25-84, 173-189
    m = one_vertex_model(Z_ONLY, (0.0, 0.0, -100.0))
    m.set_axis_scale(2, 10.0)
    m.apply_parameters([5.0])
    np.testing.assert_allclose(m.positions()[0], [0.0, 0.0, 50.0])
    m = one_vertex_model(XY_FREE)
    m.apply_parameters([100.0, 200.0])
    np.testing.assert_allclose(m.positions()[0], [100.0, 200.0, 30.0])


def test_bounds_depth_and_scaling():
    # test_dof_system.cpp:122-171
    m = Model()
    m.add_group(0, 1.0)
    m.set_group_mesh(0, np.array([[0, 0, -100.0], [0, 0, -200.0]]), np.array([[0, 1, 0]]), [Z_ONLY, XYZ_FREE])
    m.set_depth_bounds(-500.0, 50.0)
    lo, hi = m.bounds()
    assert len(lo) == 4
    assert lo[0] == -500.0 and hi[0] == 50.0
    assert lo[3] == -500.0 and hi[3] == 50.0
    assert lo[1] == -1e12 and hi[1] == 1e12  # model-level X bounds without applyModelBounds
    m2 = one_vertex_model(Z_ONLY, (0, 0, -100.0))
    m2.set_depth_bounds(-1000.0, 100.0)
    m2.set_axis_scale(2, 10.0)
    lo, hi = m2.bounds()
    assert lo[0] == -100.0 and hi[0] == 10.0


def two_box_model():
    """Two unit boxes sharing the face x = 1 (test_no_gap.cpp:43-133 style)."""
    def box(x0):
        V = np.array([[x0 + i, j, -k] for k in (0, 1) for j in (0, 1) for i in (0, 1)], float)
        F = np.array([[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1],
                      [2, 3, 7], [2, 7, 6], [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]], np.int32)
        return V, F
    m = Model()
    m.add_group(0, 2.0)
    m.add_group(1, 2.5)
    for g, x0 in enumerate((0.0, 1.0)):
        V, F = box(x0)
        m.set_group_mesh(g, V, F, Z_ONLY)
    m.build_shared_vertex_sync()
    return m


def test_global_dof_dedup_and_no_gap():
    # test_global_dofs.cpp:21-58: shared contact vertices share one global DOF
    m = two_box_model()
    inf = m.info()
    assert inf.n_vertices == 16
    assert m.n_dofs == 12  # 8 + 8 vertices, 4 shared positions
    t = m.tables()
    shared = [d for d in range(m.n_dofs) if t["dof_off"][d + 1] - t["dof_off"][d] == 2]
    assert len(shared) == 4
    x = m.assemble_parameters() + np.arange(m.n_dofs) * 0.1
    m.apply_parameters(x)
    pos = m.positions()
    for d in shared:
        a, b = t["ref_vertex"][t["dof_off"][d]:t["dof_off"][d + 1]]
        np.testing.assert_array_equal(pos[a], pos[b])
    # assembleParameterVector round trip (test_global_dofs.cpp:94-124)
    np.testing.assert_array_equal(m.assemble_parameters(), x)


def test_invalid_mesh_rejected():
    m = Model()
    m.add_group(0, 1.0)
    with pytest.raises(LithoError):
        m.set_group_mesh(0, np.zeros((3, 3)), np.array([[0, 1, 5]]), Z_ONLY)
    with pytest.raises(LithoError):
        m.set_group_mesh(0, np.array([[0, 0, np.nan], [1, 0, 0], [0, 1, 0]]), np.array([[0, 1, 2]]), Z_ONLY)
    with pytest.raises(LithoError):
        m.add_group(0, 2.0)  # duplicate id


def test_regular_grid_control_points():
    # SurfaceMesh::setControlPointStride on an N x N grid (surface_mesh.cpp:319-431)
    n = 9
    g = np.array([[i * 10.0, j * 10.0, -50.0] for j in range(n) for i in range(n)])
    tris = []
    for j in range(n - 1):
        for i in range(n - 1):
            a, b, c, d = j * n + i, j * n + i + 1, (j + 1) * n + i + 1, (j + 1) * n + i
            tris += [[a, b, c], [a, c, d]]
    m = Model()
    m.add_group(0, 1.0)
    m.set_group_mesh(0, g, np.array(tris), Z_ONLY)
    ncp = m.set_mesh_control_point_stride(0, 4)
    assert ncp == 9  # rows/cols 0, 4, 8
    assert m.n_dofs == 9
    x = np.full(9, -60.0)
    m.apply_parameters(x)
    np.testing.assert_allclose(m.positions()[:, 2], -60.0)  # bilinear of a constant is the constant
