"""Invalid, empty and ragged mesh descriptions are rejected by cfd_create with a status and a
message before any device is touched (CPU; no GPU needed).

The descriptor is the reference's mesh layout (ghost ids after the NP physical cells, 4 face
slots per cell, boundary entries (kind, cell, face, ghost)); each case below changes one field of
a valid 8 x 2 box and checks the status cfd_create returns.
"""
import ctypes

import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb

P_INT = ctypes.POINTER(ctypes.c_int)
P_DBL = ctypes.POINTER(ctypes.c_double)


class Desc:
    """A writable copy of a mesh's descriptor arrays (kept alive with the ctypes struct)."""

    def __init__(self, m):
        self.NP, self.NG = m.n_physical, m.n_ghost
        self.n_faces = m.n_faces.astype(np.int32).copy()
        self.neighbours = m.neighbours.astype(np.int32).copy()
        self.face_normals = m.face_normals.copy()
        self.face_lengths = m.face_lengths.copy()
        self.center_distances = m.center_distances.copy()
        self.center_vectors = m.center_vectors.copy()
        self.area = m.area.copy()
        self.inv_area = m.inv_area.copy()
        self.boundary = m.boundary.astype(np.int32).copy()
        self.NB = len(self.boundary)
        self.drop = set()

    def struct(self):
        def ip(a, name):
            return ctypes.cast(None, P_INT) if name in self.drop else a.ctypes.data_as(P_INT)

        def dp(a, name):
            return ctypes.cast(None, P_DBL) if name in self.drop else a.ctypes.data_as(P_DBL)

        d = cb.MeshDesc()
        d.n_physical, d.n_ghost, d.n_boundary = self.NP, self.NG, self.NB
        d.n_faces = ip(self.n_faces, "n_faces")
        d.neighbours = ip(self.neighbours, "neighbours")
        d.face_normals = dp(self.face_normals, "face_normals")
        d.face_lengths = dp(self.face_lengths, "face_lengths")
        d.center_distances = dp(self.center_distances, "center_distances")
        d.center_vectors = dp(self.center_vectors, "center_vectors")
        d.area = dp(self.area, "area")
        d.inv_area = dp(self.inv_area, "inv_area")
        d.boundary = ip(self.boundary, "boundary")
        return d


def create_status(desc, **cfg):
    d = desc.struct()
    c = cb.default_config(**cfg)
    h = ctypes.c_void_p()
    s = cb.lib().cfd_create(ctypes.byref(d), ctypes.byref(c), ctypes.byref(h))
    if s == cb.CFD_OK:
        cb.lib().cfd_destroy(h)
    return s, cb.lib().cfd_last_error().decode()


@pytest.fixture()
def desc():
    return Desc(cb.Mesh.box(8, 2))


def test_empty_mesh_is_bad_arg(desc):
    desc.NP = 0
    s, msg = create_status(desc)
    assert s == cb.CFD_ERR_BAD_ARG and "sizes" in msg


def test_negative_counts_are_bad_arg(desc):
    desc.NG = -1
    assert create_status(desc)[0] == cb.CFD_ERR_BAD_ARG
    desc.NG = Desc(cb.Mesh.box(8, 2)).NG
    desc.NB = -3
    assert create_status(desc)[0] == cb.CFD_ERR_BAD_ARG


@pytest.mark.parametrize("name", ["n_faces", "neighbours", "face_normals", "face_lengths", "area", "inv_area",
                                  "boundary"])
def test_missing_array_is_bad_arg(desc, name):
    desc.drop.add(name)
    s, msg = create_status(desc)
    assert s == cb.CFD_ERR_BAD_ARG and "missing" in msg, (name, msg)


def test_second_order_needs_centre_distances(desc):
    desc.drop.add("center_distances")
    s, msg = create_status(desc, is_second_order=1)
    assert s == cb.CFD_ERR_BAD_ARG and "centre distances" in msg


@pytest.mark.parametrize("nf", [0, 2, 5, -1])
def test_ragged_cell_outside_three_or_four_faces_is_a_mesh_error(desc, nf):
    desc.n_faces[5] = nf
    s, msg = create_status(desc)
    assert s == cb.CFD_ERR_MESH and "cell 5" in msg


@pytest.mark.parametrize("bad", [-1, "NT"])
def test_neighbour_out_of_range_is_a_mesh_error(desc, bad):
    desc.neighbours[3, 1] = desc.NP + desc.NG if bad == "NT" else bad
    s, msg = create_status(desc)
    assert s == cb.CFD_ERR_MESH and "cell 3" in msg and "neighbour" in msg


@pytest.mark.parametrize("field,value", [(0, 4), (0, -1), (1, -1), (1, "NP"), (2, 4), (3, 0), (3, "NT")])
def test_bad_boundary_entry_is_a_mesh_error(desc, field, value):
    v = {"NP": desc.NP, "NT": desc.NP + desc.NG}.get(value, value)
    desc.boundary[2, field] = v
    s, msg = create_status(desc)
    assert s == cb.CFD_ERR_MESH and "boundary entry 2" in msg, (field, value, msg)


def test_triangle_with_a_fourth_slot_is_accepted_up_to_the_device():
    """A ragged (mixed triangle / quad) mesh passes validation; without a device the call then
    stops at the device check, not at the mesh."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    m = cb.Mesh.bump(20, 8, 3.0, 1.0, 0.1, 2, 0.3, 7, True)
    d = Desc(m)
    assert (d.n_faces == 3).any() and (d.n_faces == 4).any()
    assert create_status(d)[0] == cb.CFD_ERR_NO_DEVICE
    assert create_status(Desc(cb.Mesh.box(8, 2)))[0] == cb.CFD_ERR_NO_DEVICE
