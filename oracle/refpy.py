"""Test infrastructure only: ctypes bindings of the two CPU checkers.

  RefRun    oracle/_ref/libcfdref.so — the reference's own CPU code (see ref_harness.cpp)
  OracleRun oracle/_build/liboracle.so — the plain-C restatement (cfd_oracle.c)

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg only.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libcfdref.so")
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
# The reference checkout: CFD_REFERENCE_DIR, else a directory "reference" beside this repository.
REF_SRC = os.environ.get("CFD_REFERENCE_DIR", os.path.abspath(os.path.join(HERE, "..", "..", "reference")))

_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)


def _dp(a):
    return a.ctypes.data_as(_DP)


def _ip(a):
    return a.ctypes.data_as(_IP)


def build_oracle():
    """Compiles the C restatement (needs only gcc)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
    return ORACLE_LIB


def build_ref():
    """Compiles the reference CPU path from its sources when they are present."""
    if not os.path.isdir(os.path.join(REF_SRC, "src")):
        return None
    subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "ref", "REF=" + REF_SRC])
    return REF_LIB


def ref_available():
    return os.path.exists(REF_LIB)


REFCUDA_LIB = os.path.join(HERE, "_ref", "librefcuda.so")


def build_refcuda():
    """Compiles the reference's GPU flux kernels from their sources when they are present."""
    if not os.path.isdir(os.path.join(REF_SRC, "CUDA_KERNELS")):
        return None
    subprocess.check_call(["make", "-s", "-C", HERE, "refcuda", "REF=" + REF_SRC])
    return REFCUDA_LIB


def refcuda_available():
    return os.path.exists(REFCUDA_LIB)


def refcuda_hllc(U, P6, nbr, normals, areas, flux, num_cells):
    """Runs the reference's hllc_flux_kernel (its launch_hllc_flux) on device arrays given as
    integer data pointers; returns the CUDA status (0 = success)."""
    L = ctypes.CDLL(REFCUDA_LIB)
    L.refcu_hllc_flux.restype = ctypes.c_int
    L.refcu_hllc_flux.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int]
    return L.refcu_hllc_flux(U, P6, nbr, normals, areas, flux, num_cells)


def refcuda_flux_launcher(scheme):
    """The launch-only entry of the reference's roe_flux_kernel ("roe") or hllc_flux_kernel
    ("hllc") on device arrays given as integer data pointers (legacy default stream, no
    synchronisation); returns a callable (U, P6, nbr, normals, areas, flux, num_cells) -> status."""
    L = ctypes.CDLL(REFCUDA_LIB)
    fn = getattr(L, "refcu_%s_flux_launch" % scheme)
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int]
    return fn


_refcu = []


def _refcu_lib():
    if not _refcu:
        L = ctypes.CDLL(REFCUDA_LIB)
        L.refcu_limiter.argtypes = [ctypes.c_int, _DP, _DP, ctypes.c_int, _DP]
        L.refcu_ausm_flux.argtypes = [_DP, _DP, _DP, _DP, ctypes.c_int, _DP]
        L.refcu_farfield.argtypes = [_DP, _DP, ctypes.c_int] + [ctypes.c_double] * 4
        L.refcu_rk_stage.argtypes = [ctypes.c_int, ctypes.c_int, _DP, _DP, _DP, _DP, _DP, ctypes.c_double,
                                     ctypes.c_int]
        for n in ("refcu_limiter", "refcu_ausm_flux", "refcu_farfield", "refcu_rk_stage"):
            getattr(L, n).restype = ctypes.c_int
        _refcu.append(L)
    return _refcu[0]


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def refcuda_limiter(kind, a, b):
    """phi(a, b) of the reference's vanleer/superbee/vanalbada_limiter_device (kind 2/3/4)."""
    a, b = _c(a), _c(b)
    out = np.zeros_like(a)
    rc = _refcu_lib().refcu_limiter(kind, _dp(a), _dp(b), a.size, _dp(out))
    if rc:
        raise RuntimeError("refcu_limiter: CUDA error %d" % rc)
    return out


def refcuda_ausm_flux(UL5, UR5, normals3, areas):
    """The reference's ausm_flux_kernel on 5-component states; returns fluxes [n, 5]."""
    UL5, UR5, normals3, areas = _c(UL5), _c(UR5), _c(normals3), _c(areas)
    out = np.zeros((UL5.shape[0], 5))
    rc = _refcu_lib().refcu_ausm_flux(_dp(UL5), _dp(UR5), _dp(normals3), _dp(areas), UL5.shape[0], _dp(out))
    if rc:
        raise RuntimeError("refcu_ausm_flux: CUDA error %d" % rc)
    return out


def refcuda_farfield(U4, normals8, rho_inf, u_inf, v_inf, p_inf):
    """The reference's farfield_bc_kernel: boundary states [n, 4] from interior states [n, 4]."""
    U = _c(U4).copy()
    normals8 = _c(normals8)
    rc = _refcu_lib().refcu_farfield(_dp(U), _dp(normals8), U.shape[0], rho_inf, u_inf, v_inf, p_inf)
    if rc:
        raise RuntimeError("refcu_farfield: CUDA error %d" % rc)
    return U


def refcuda_rk_stage(which, stage, U5, T1, T2, net_flux5, volumes, dt):
    """One stage of the reference's tvd_rk3_kernel (which 3) or rk4_complete_kernel (which 4);
    U5, T1, T2 ([n, 5] float64 C arrays) are updated in place."""
    F, V = _c(net_flux5), _c(volumes)
    rc = _refcu_lib().refcu_rk_stage(which, stage, _dp(U5), _dp(T1), _dp(T2), _dp(F), _dp(V), dt, U5.shape[0])
    if rc:
        raise RuntimeError("refcu_rk_stage: CUDA error %d" % rc)


_ref = {}
DROPIN_LIB = os.path.join(HERE, "_ref", "libcfdref_dropin.so")


def build_dropin():
    """The reference solver linked with the B200 drop-in shim (needs the reference sources and
    libcfd_b200.so)."""
    if not os.path.isdir(os.path.join(REF_SRC, "src")):
        return None
    subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "dropin", "REF=" + REF_SRC])
    return DROPIN_LIB


def reflib(path=REF_LIB):
    if path not in _ref:
        L = ctypes.CDLL(path)
        for n in ["refh_reset", "refh_clear_boundary_lists", "refh_apply_bc", "refh_net_flux", "refh_explicit",
                  "refh_rk3", "refh_estimate_error", "refh_update", "refh_ausm_net_flux", "refh_exit_fixed_p",
                  "refh_lax_friedrichs"]:
            getattr(L, n).restype = None
        L.refh_load_vtk.argtypes = [ctypes.c_char_p]
        L.refh_load_vtk.restype = ctypes.c_int
        L.refh_add_boundary.argtypes = [ctypes.c_int] * 4
        L.refh_finalize_mesh.restype = ctypes.c_int
        L.refh_counts.argtypes = [_IP]
        L.refh_get_boundary_list.argtypes = [ctypes.c_int, _IP]
        L.refh_get_geometry.argtypes = [_IP, _IP, _DP, _DP, _DP, _DP, _DP, _DP]
        L.refh_set_param.argtypes = [ctypes.c_char_p, ctypes.c_double]
        L.refh_set_param.restype = ctypes.c_int
        L.refh_set_state.argtypes = [_DP, ctypes.c_int]
        for n in ["refh_get_U", "refh_get_prim", "refh_get_net_flux", "refh_get_delU", "refh_get_dt",
                  "refh_get_error"]:
            getattr(L, n).argtypes = [_DP]
        L.refh_get_rk_states.argtypes = [_DP, _DP]
        for n in ["refh_min_dt", "refh_total_time", "refh_get_min_dt"]:
            getattr(L, n).restype = ctypes.c_double
        L.refh_iterations.restype = ctypes.c_int
        L.refh_iterate.argtypes = [ctypes.c_int, ctypes.c_double]
        L.refh_iterate.restype = ctypes.c_int
        L.refh_gradient.argtypes = [ctypes.c_int, _DP]
        L.refh_amr.argtypes = [ctypes.c_double, ctypes.c_double, _DP, ctypes.POINTER(ctypes.c_uint8)]
        L.refh_write_solution.argtypes = [ctypes.c_char_p]
        L.refh_read_write_grid.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.refh_append_solution.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        for n in ("refh_write_solution", "refh_read_write_grid", "refh_append_solution"):
            getattr(L, n).restype = None
        _ref[path] = L
    return _ref[path]


class RefRun:
    """The reference CPU path on one mesh (process-global state: one instance at a time)."""

    def __init__(self, mesh, params, lib_path=REF_LIB):
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "mesh.vtk")
            mesh.write_vtk(path)
            # Boundary lists from the mesh layer (identical to the bounding-box lists on box domains).
            self._setup(path, mesh.boundary, params, lib_path)
        if self.NP != mesh.n_physical:
            raise RuntimeError("reference reader returned %d cells, expected %d" % (self.NP, mesh.n_physical))

    @classmethod
    def from_vtk(cls, path, boundary, params, lib_path=REF_LIB):
        """The reference path on a VTK file read by its own reader.  boundary: (kind, cell, face,
        ghost) rows replacing the reader's bounding-box lists, or None to keep them."""
        self = cls.__new__(cls)
        self._setup(path, boundary, params, lib_path)
        return self

    def _setup(self, path, boundary, params, lib_path):
        L = reflib(lib_path)
        np_ = L.refh_load_vtk(path.encode())
        if np_ <= 0:
            raise RuntimeError("the reference reader could not read %s" % path)
        if boundary is not None:
            L.refh_clear_boundary_lists()
            for kind, c, f, g in boundary:
                L.refh_add_boundary(int(kind), int(c), int(f), int(g))
        for k, v in params.items():
            if L.refh_set_param(k.encode(), float(v)) != 0:
                raise KeyError(k)
        self.NT = L.refh_finalize_mesh()
        self.NP = np_
        self.L = L

    def set_state(self, U):
        U = np.ascontiguousarray(U, np.float64)
        self.L.refh_set_state(_dp(U), U.shape[0])

    def geometry(self):
        NP, NT = self.NP, self.NT
        nf = np.zeros(NP, np.int32)
        nbr = np.zeros((NP, 4), np.int32)
        nrm = np.zeros((NP, 8))
        ln = np.zeros((NP, 4))
        ccd = np.zeros((NP, 4))
        ar = np.zeros(NP)
        ia = np.zeros(NP)
        cen = np.zeros((NT, 3))
        self.L.refh_get_geometry(_ip(nf), _ip(nbr), _dp(nrm), _dp(ln), _dp(ccd), _dp(ar), _dp(ia), _dp(cen))
        return dict(n_faces=nf, neighbours=nbr, face_normals=nrm, face_lengths=ln, center_distances=ccd, area=ar,
                    inv_area=ia, centers=cen)

    def boundary_lists(self):
        cnt = np.zeros(6, np.int32)
        self.L.refh_counts(_ip(cnt))
        out = []
        for kind in range(4):
            a = np.zeros(max(1, 3 * cnt[2 + kind]), np.int32)
            self.L.refh_get_boundary_list(kind, _ip(a))
            out.append(a[:3 * cnt[2 + kind]].reshape(-1, 3))
        return out

    def state(self):
        NP, NT = self.NP, self.NT
        U = np.zeros((NT, 4))
        P = np.zeros((NT, 11))
        dt = np.zeros(NP)
        net = np.zeros((NP, 4))
        dU = np.zeros((NP, 4))
        self.L.refh_get_U(_dp(U))
        self.L.refh_get_prim(_dp(P))
        self.L.refh_get_dt(_dp(dt))
        self.L.refh_get_net_flux(_dp(net))
        self.L.refh_get_delU(_dp(dU))
        return {"U": U, "prim": P, "dt": dt, "net_flux": net, "delU": dU}

    def rk_states(self):
        u1 = np.zeros((self.NP, 4))
        u2 = np.zeros((self.NP, 4))
        self.L.refh_get_rk_states(_dp(u1), _dp(u2))
        return u1, u2

    def error(self):
        e = np.zeros(4)
        self.L.refh_get_error(_dp(e))
        return e

    def iterate(self, n, t_end=0.0):
        return self.L.refh_iterate(n, t_end)

    def min_dt(self):
        return self.L.refh_min_dt()

    def total_time(self):
        return self.L.refh_total_time()

    def gradient(self, var):
        g = np.zeros((self.NP, 2))
        self.L.refh_gradient(var, _dp(g))
        return g

    def amr(self, threshold, max_fraction):
        ind = np.zeros(self.NP)
        tags = np.zeros(self.NP, np.uint8)
        self.L.refh_amr(threshold, max_fraction, _dp(ind), tags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        return ind, tags


class _OrcConfig(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ["dissipation_type", "is_second_order", "time_accurate",
                                            "local_time_stepping", "integrator", "limiter", "reconstruct_primitive",
                                            "muscl", "precision", "inlet_bc", "exit_bc"]] + \
               [(n, ctypes.c_double) for n in ["cfl", "zeta", "zeta1", "inlet_rho", "inlet_p", "inlet_p0", "inlet_t0",
                                               "exit_p", "r_gas", "inlet_u", "inlet_v"]] + \
               [(n, ctypes.c_int) for n in ["weno", "weno_char"]] + [("ef_linear", ctypes.c_double),
                                                                            ("shock_fix", ctypes.c_double)] + \
               [(n, ctypes.c_int) for n in ["movers_single", "movers_efix"]]


_orc = None


def oraclelib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            build_oracle()
        L = ctypes.CDLL(ORACLE_LIB)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, ctypes.c_int, _IP, _IP, _DP, _DP, _DP, _DP, _DP, _DP, ctypes.c_int,
                                 _IP, ctypes.POINTER(_OrcConfig)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_state.argtypes = [ctypes.c_void_p, _DP, ctypes.c_int]
        for n in ["orc_apply_bc", "orc_net_flux", "orc_rk", "orc_estimate_error", "orc_update"]:
            getattr(L, n).argtypes = [ctypes.c_void_p]
            getattr(L, n).restype = None
        L.orc_explicit.argtypes = [ctypes.c_void_p]
        L.orc_iterate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.orc_get.argtypes = [ctypes.c_void_p, _DP, _DP, _DP, _DP, _DP]
        L.orc_get_stage.argtypes = [ctypes.c_void_p, _DP]
        for n in ["orc_min_dt", "orc_total_time"]:
            getattr(L, n).argtypes = [ctypes.c_void_p]
            getattr(L, n).restype = ctypes.c_double
        L.orc_error.argtypes = [ctypes.c_void_p, _DP]
        L.orc_gradient.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
        L.orc_amr.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _DP, ctypes.POINTER(ctypes.c_uint8)]
        L.orc_bad_cell.argtypes = [ctypes.c_void_p]
        _orc = L
    return _orc


class OracleRun:
    """The C restatement on one mesh; params use the solver-config field names."""

    def __init__(self, mesh, **params):
        L = oraclelib()
        c = _OrcConfig()
        c.dissipation_type = params.get("dissipation_type", 3)
        c.is_second_order = params.get("is_second_order", 0)
        c.time_accurate = params.get("time_accurate", 1)
        c.local_time_stepping = params.get("local_time_stepping", 0)
        c.integrator = params.get("integrator", 0)
        c.limiter = params.get("limiter", 0)
        c.reconstruct_primitive = params.get("reconstruct_primitive", 0)
        c.muscl = params.get("muscl", 0)
        c.precision = params.get("precision", 0)
        c.inlet_bc = params.get("inlet_bc", 0)
        c.exit_bc = params.get("exit_bc", 0)
        c.cfl = params.get("cfl", 0.5)
        c.zeta = params.get("limiter_zeta", 0.5)
        c.zeta1 = params.get("limiter_zeta1", 0.5)
        c.inlet_rho = params.get("inlet_rho", 1.0)
        c.inlet_p = params.get("inlet_p", 1.0)
        c.inlet_p0 = params.get("inlet_p0", 0.0)
        c.inlet_t0 = params.get("inlet_t0", 0.0)
        c.exit_p = params.get("exit_p", 0.0)
        c.r_gas = params.get("r_gas", 287.0)
        c.inlet_u = params.get("inlet_u", 0.0)
        c.inlet_v = params.get("inlet_v", 0.0)
        c.weno = params.get("weno", 0)
        c.weno_char = params.get("weno_characteristic", 0)
        c.ef_linear = params.get("entropy_fix_linear", 0.0)
        c.shock_fix = params.get("shock_fix", 0.0)
        c.movers_single = params.get("movers_single_alpha", 0)
        c.movers_efix = params.get("movers_entropy_fix", 0)
        self.m = mesh
        self._keep = [np.ascontiguousarray(a) for a in (
            mesh.n_faces.astype(np.int32), mesh.neighbours.astype(np.int32), mesh.face_normals, mesh.face_lengths,
            mesh.center_distances, mesh.center_vectors, mesh.area, mesh.inv_area,
            mesh.boundary.astype(np.int32).reshape(-1))]
        k = self._keep
        self.h = L.orc_create(mesh.n_physical, mesh.n_ghost, _ip(k[0]), _ip(k[1]), _dp(k[2]), _dp(k[3]), _dp(k[4]),
                              _dp(k[5]), _dp(k[6]), _dp(k[7]), mesh.boundary.shape[0], _ip(k[8]), ctypes.byref(c))
        self.L = L
        self.NP, self.NT = mesh.n_physical, mesh.n_total

    def __del__(self):
        try:
            self.L.orc_destroy(self.h)
        except Exception:
            pass

    def set_state(self, U):
        U = np.ascontiguousarray(U, np.float64)
        self.L.orc_set_state(self.h, _dp(U), U.shape[0])

    def state(self):
        NP, NT = self.NP, self.NT
        out = {"U": np.zeros((NT, 4)), "prim": np.zeros((NT, 11)), "dt": np.zeros(NP), "net_flux": np.zeros((NP, 4)),
               "delU": np.zeros((NP, 4))}
        self.L.orc_get(self.h, _dp(out["U"]), _dp(out["prim"]), _dp(out["dt"]), _dp(out["net_flux"]), _dp(out["delU"]))
        return out

    def stage_state(self):
        S = np.zeros((self.NP, 4))
        self.L.orc_get_stage(self.h, _dp(S))
        return S

    def iterate(self, n, t_end=0.0):
        return self.L.orc_iterate(self.h, n, t_end)

    def apply_bc(self):
        self.L.orc_apply_bc(self.h)

    def net_flux(self):
        self.L.orc_net_flux(self.h)

    def explicit(self):
        return self.L.orc_explicit(self.h)

    def lax_friedrichs(self):
        return self.L.orc_lax_friedrichs(self.h)

    def rk(self):
        self.L.orc_rk(self.h)

    def estimate_error(self):
        self.L.orc_estimate_error(self.h)
        return self.error()

    def update(self):
        self.L.orc_update(self.h)

    def error(self):
        e = np.zeros(4)
        self.L.orc_error(self.h, _dp(e))
        return e

    def min_dt(self):
        return self.L.orc_min_dt(self.h)

    def total_time(self):
        return self.L.orc_total_time(self.h)

    def gradient(self, slot):
        g = np.zeros((self.NP, 2))
        self.L.orc_gradient(self.h, slot, _dp(g))
        return g

    def amr(self, threshold, max_fraction):
        ind = np.zeros(self.NP)
        tags = np.zeros(self.NP, np.uint8)
        self.L.orc_amr(self.h, threshold, max_fraction, _dp(ind), tags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        return ind, tags
