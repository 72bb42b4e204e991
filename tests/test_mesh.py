"""Mesh layer: generators + the reference's ingest rules, checked against fixtures produced by the
reference's own reader (src/Read_Gmsh_File.cpp:11-402, src/Grid_Computations.cpp:394-827)."""
import os

import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb
from cases import CASES, make_mesh
from conftest import assert_bits_equal, load_golden

from oracle.refpy import REF_SRC as REF_DIR  # CFD_REFERENCE_DIR, else "reference" beside the repository


@pytest.mark.parametrize("name", sorted(CASES))
def test_geometry_matches_reference_reader(name):
    g = load_golden(name)
    m = make_mesh(CASES[name])
    for k in ("neighbours", "face_normals", "face_lengths", "center_distances", "area", "inv_area", "centers"):
        assert_bits_equal(getattr(m, k), g["geo_" + k], name + ":" + k)


def test_ghost_numbering_cell_major_face_minor():
    m = cb.Mesh.box(5, 3)
    ghosts = []
    for c in range(m.n_physical):
        for f in range(m.n_faces[c]):
            if m.neighbours[c, f] >= m.n_physical:
                ghosts.append(m.neighbours[c, f])
    assert ghosts == list(range(m.n_physical, m.n_total))
    assert sorted(m.boundary[:, 3]) == ghosts


def test_box_face_order_and_bbox_classification():
    # Anticlockwise sort from the vertex average puts the bottom edge first on axis-aligned quads.
    m = cb.Mesh.box(4, 2, 0.0, 1.0, 0.0, 0.5)
    assert np.allclose(m.face_normals[0], [0, -1, 1, 0, 0, 1, -1, 0])
    kinds = {int(k): set() for k in range(4)}
    for kind, c, f, g in m.boundary:
        kinds[int(kind)].add((int(c), int(f)))
    assert len(kinds[cb.BC_INLET]) == 2 and len(kinds[cb.BC_EXIT]) == 2 and len(kinds[cb.BC_WALL]) == 8


def test_vtk_round_trip(tmp_path):
    m = cb.Mesh.bump(20, 10, thickness=0.1, n_quad_layers=2, jitter=0.3, seed=3)
    p = str(tmp_path / "m.vtk")
    m.write_vtk(p)
    r = cb.Mesh.read_vtk(p)
    # The reader uses the bounding-box classification; geometry and connectivity are unchanged.
    for k in ("neighbours", "face_normals", "face_lengths", "center_distances", "area", "inv_area"):
        assert_bits_equal(getattr(m, k), getattr(r, k), k)


def test_half_cylinder_boundary_kinds():
    m = cb.Mesh.half_cylinder(16, 8)
    counts = np.bincount(m.boundary[:, 0], minlength=4)
    assert counts[cb.BC_WALL] == 16 and counts[cb.BC_INLET] == 16 and counts[cb.BC_EXIT] == 16
    assert m.n_ghost == 48
    assert np.all(m.area > 0)


def test_mixed_mesh_has_triangles_and_quads():
    m = cb.Mesh.bump(30, 16, n_quad_layers=4, triangles=True)
    assert set(np.unique(m.n_faces)) == {3, 4}
    assert (m.n_faces == 4).sum() == 30 * 8


def test_mesh_errors_are_status_codes():
    with pytest.raises(cb.CfdError):
        cb.Mesh.box(0, 4)
    with pytest.raises(cb.CfdError):
        cb.Mesh.read_vtk("/nonexistent/mesh.vtk")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "Grid_Files")), reason="reference grids not present")
def test_shipped_ramp_grid_known_answers():
    """TEST_SUMMARY.md:48-100 of the reference pins Ramp_15o_52_18.vtk: 800 quads, total area
    5.397113, min/max area 0.004434/0.008255, 16 inlet and 16 exit faces.  Its ghost count (131)
    predates the face-ordered reader: the reference's current Read_VTK_Grid builds 132 ghosts
    (16 inlet + 16 exit + 100 wall), which is what the mesh layer must reproduce.  Its areas are
    the diagonal cross product |d1 x d2| of the older Construct_Cell (src/Grid_Computations.cpp:
    507-515), i.e. twice the shoelace area the current reader stores (:547-557)."""
    path = None
    for dp, _, fs in os.walk(os.path.join(REF_DIR, "Grid_Files")):
        for f in fs:
            if f == "Ramp_15o_52_18.vtk":
                path = os.path.join(dp, f)
    if path is None:
        pytest.skip("Ramp_15o_52_18.vtk not found")
    m = cb.Mesh.read_vtk(path)
    assert m.n_physical == 800
    assert m.n_ghost == 132
    counts = np.bincount(m.boundary[:, 0], minlength=4)
    assert list(counts) == [16, 16, 100, 0]
    assert abs(2 * m.area.sum() - 5.397113) < 5e-7
    assert abs(2 * m.area.min() - 0.004434) < 5e-7 and abs(2 * m.area.max() - 0.008255) < 5e-7
    from oracle import refpy
    if refpy.ref_available():
        r = refpy.RefRun(m, {"CFL": 0.5})
        g = r.geometry()
        for k in ("neighbours", "face_normals", "face_lengths", "center_distances", "area", "inv_area"):
            assert_bits_equal(getattr(m, k), g[k], k)


def test_ramp_boundary_kinds():
    """Generated ramps: the bounding-box rule (top = wall) by default, an open top on request."""
    nx, ny = 8, 4
    for open_top, want in ((False, [ny, ny, 2 * nx]), (True, [ny, ny + nx, nx])):
        m = cb.Mesh.ramp(nx, ny, 3.0, 1.0, 1.0, 15.0, open_top=open_top)
        kinds = np.bincount(m.boundary[:, 0], minlength=3)
        assert kinds.tolist() == want, (open_top, kinds)
        assert m.n_physical == nx * ny and m.n_ghost == 2 * (nx + ny)
