"""Test infrastructure only: the half-cylinder O-grid written as a legacy VTK file with numpy and
the C library (no product code), and the reference's own CPU solver set up on it.

Used by bench.py's CPU-baseline leg and its --impl reference arm, so that the timed reference run
maps none of the product's libraries.  The grid is the body-fitted O-grid of the M = 3 half-cylinder
case: theta in [pi/2, 3pi/2] (the front half, facing -x), body radius r_body, outer radius
r_outer, geometric radial stretching `ratio`; cell (i, j) is number j * ntheta + i.  The point
coordinates repeat the product's generator operation by operation (libm pow, cos and sin through
Python's math module), so the file is the one the product's writer produces.

Boundary kinds (harness codes 0 inlet, 1 exit, 2 wall): the body is a slip wall, the outer arc a
supersonic inlet, the two radial cut lines on x = 0 extrapolation exits.  The reference's VTK reader
(Read_VTK_Grid, src/Read_Gmsh_File.cpp:11) numbers the ghost cells; its own bounding-box
classification does not fit a curved domain, so each boundary face is classified here from the
reader's face normal against the radial direction at the cell centre.
"""
import math
import os
import tempfile

import numpy as np

from oracle import refpy

GAMMA = 1.4


def half_cylinder_points(ntheta, nr, r_body, r_outer, ratio):
    """Node coordinates [(ntheta + 1) * (nr + 1), 3], node (i, j) at j * (ntheta + 1) + i."""
    denom = float(nr) if ratio == 1.0 else (math.pow(ratio, nr) - 1.0)
    r = []
    for j in range(nr + 1):
        s = (j / denom) if ratio == 1.0 else (math.pow(ratio, j) - 1.0) / denom
        r.append(r_body + (r_outer - r_body) * s)
    r[nr] = r_outer
    pi = 3.14159265358979323846
    cos_t, sin_t = [], []
    for i in range(ntheta + 1):
        th = 0.5 * pi + pi * (float(i) / ntheta)
        cos_t.append(math.cos(th))
        sin_t.append(math.sin(th))
    R = np.array(r)[:, None]
    x = R * np.array(cos_t)[None, :]
    y = R * np.array(sin_t)[None, :]
    x[:, 0] = 0.0
    x[:, ntheta] = 0.0
    return np.stack([x.ravel(), y.ravel(), np.zeros(x.size)], axis=1)


def write_half_cylinder_vtk(path, ntheta, nr, r_body=1.0, r_outer=4.0, ratio=1.005):
    """Legacy ASCII VTK unstructured grid of quads (cell type 9), nodes of cell (i, j) in the
    order (i, j), (i+1, j), (i+1, j+1), (i, j+1)."""
    pts = half_cylinder_points(ntheta, nr, r_body, r_outer, ratio)
    i = np.tile(np.arange(ntheta), nr)
    j = np.repeat(np.arange(nr), ntheta)
    P = lambda a, b: b * (ntheta + 1) + a
    cells = np.stack([np.full(i.size, 4), P(i, j), P(i + 1, j), P(i + 1, j + 1), P(i, j + 1)], axis=1)
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 2.0\ncfd-b200 mesh\nASCII\nDATASET UNSTRUCTURED_GRID\n")
        f.write("POINTS %d double\n" % len(pts))
        f.write("".join("%.17g %.17g %.17g\n" % tuple(p) for p in pts))
        f.write("CELLS %d %d\n" % (len(cells), cells.size))
        np.savetxt(f, cells, fmt="%d")
        f.write("CELL_TYPES %d\n" % len(cells))
        f.write("9\n" * len(cells))


def classify_boundary(geo, n_physical):
    """(kind, cell, face, ghost) rows for every face whose neighbour is a ghost cell, from the
    reader's neighbours and normals: normal against the radial unit vector at the cell centre,
    < -0.5 body wall (2), > 0.5 outer-arc inlet (0), else a cut-line exit (1)."""
    nbr, nrm, cen = geo["neighbours"], geo["face_normals"], geo["centers"]
    rows = []
    for c in range(n_physical):
        cx, cy = cen[c, 0], cen[c, 1]
        rr = math.hypot(cx, cy)
        for f in range(geo["n_faces"][c]):
            g = int(nbr[c, f])
            if g < n_physical:
                continue
            d = (nrm[c, 2 * f] * cx + nrm[c, 2 * f + 1] * cy) / rr
            kind = 2 if d < -0.5 else 0 if d > 0.5 else 1
            rows.append((kind, c, f, g))
    return rows


def reference_half_cylinder(ntheta, nr, r_body, r_outer, ratio, params, mach=3.0, rho=1.0, p=1.0 / GAMMA,
                            lib_path=None):
    """The reference's CPU solver (oracle/_ref/libcfdref.so, or the library at lib_path, e.g. the
    reference linked with the B200 drop-in) set up on the O-grid with the given Solver_Config
    parameters, at a uniform freestream state (rho, u = mach * a, v = 0, p) on every physical and
    ghost row.  Returns the refpy.RefRun."""
    lib = lib_path or refpy.REF_LIB
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "ogrid.vtk")
        write_half_cylinder_vtk(path, ntheta, nr, r_body, r_outer, ratio)
        probe = refpy.RefRun.from_vtk(path, None, {}, lib_path=refpy.REF_LIB)
        geo = probe.geometry()
        rows = classify_boundary(geo, probe.NP)
        run = refpy.RefRun.from_vtk(path, rows, params, lib_path=lib)
    u = mach * math.sqrt(GAMMA * p / rho)
    U = np.zeros((run.NT, 4))
    U[:, 0] = rho
    U[:, 1] = rho * u
    U[:, 3] = (p / (1.4 - 1.0)) + rho * (0.5 * (u * u + 0.0 * 0.0))
    run.set_state(U)
    return run
