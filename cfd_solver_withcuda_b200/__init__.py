"""B200-native explicit finite-volume residual/update path (ctypes binding of libcfd_b200.so).

The product is the C ABI in include/cfd_b200.h, implemented by the in-tree shared library
libcfd_b200.so (C++ host runtime + sm_100a CUDA kernels).  This module is a thin binding with
the reference's vocabulary (Explicit_Method, Runge_Kutta_Method, Evaluate_Cell_Net_Flux, ...);
it does no arithmetic of its own and has no CPU fallback: every solver call goes to the CUDA
library and fails loudly if it cannot be loaded or no device is present.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcfd_b200.so")

CFD_OK = 0
CFD_ERR_BAD_ARG = 1
CFD_ERR_CUDA = 2
CFD_ERR_NONPHYSICAL = 3
CFD_ERR_DT_NONPOSITIVE = 4
CFD_ERR_TIMEOUT = 5
CFD_ERR_DIVERGED = 6
CFD_ERR_MESH = 7
CFD_ERR_IO = 8
CFD_ERR_NO_DEVICE = 9
STATUS_NAMES = {0: "OK", 1: "BAD_ARG", 2: "CUDA", 3: "NONPHYSICAL", 4: "DT_NONPOSITIVE", 5: "TIMEOUT",
                6: "DIVERGED", 7: "MESH", 8: "IO", 9: "NO_DEVICE"}

BC_INLET, BC_EXIT, BC_WALL, BC_SYMMETRY = 0, 1, 2, 3
DISS_LLF, DISS_MOVERS, DISS_ROE, DISS_RICCA, DISS_MOVERS_NWSC, DISS_AUSM, DISS_HLLC, DISS_AUSM_GPU = 1, 2, 3, 4, 5, 6, 7, 8
LIM_REF_MINMOD, LIM_MINMOD, LIM_VANLEER, LIM_SUPERBEE, LIM_VANALBADA = 0, 1, 2, 3, 4
INT_REFERENCE, INT_RK4, INT_SSPRK3, INT_RK3_GPU_REF, INT_RK4_GPU_REF = 0, 1, 2, 3, 4
INLET_SUPERSONIC, INLET_SUBSONIC_REF, INLET_TOTAL_PT, INLET_FIXED, INLET_FARFIELD = 0, 1, 2, 3, 4
EXIT_SUPERSONIC, EXIT_SUBSONIC_REF, EXIT_STATIC_P, EXIT_FIXED_P_REF = 0, 1, 2, 3
PREC_FP64, PREC_FP32_FLUX = 0, 1
MUSCL_REFERENCE, MUSCL_GRADIENT = 0, 1


class CfdError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), msg))
        self.status = status


class MeshDesc(ctypes.Structure):
    _fields_ = [("n_physical", ctypes.c_int), ("n_ghost", ctypes.c_int),
                ("n_faces", ctypes.POINTER(ctypes.c_int)), ("neighbours", ctypes.POINTER(ctypes.c_int)),
                ("face_normals", ctypes.POINTER(ctypes.c_double)), ("face_lengths", ctypes.POINTER(ctypes.c_double)),
                ("center_distances", ctypes.POINTER(ctypes.c_double)),
                ("center_vectors", ctypes.POINTER(ctypes.c_double)), ("area", ctypes.POINTER(ctypes.c_double)),
                ("inv_area", ctypes.POINTER(ctypes.c_double)), ("n_boundary", ctypes.c_int),
                ("boundary", ctypes.POINTER(ctypes.c_int))]


class Config(ctypes.Structure):
    _fields_ = [("dissipation_type", ctypes.c_int), ("is_second_order", ctypes.c_int),
                ("time_accurate", ctypes.c_int), ("local_time_stepping", ctypes.c_int),
                ("integrator", ctypes.c_int), ("limiter", ctypes.c_int), ("reconstruct_primitive", ctypes.c_int),
                ("muscl", ctypes.c_int),
                ("inlet_bc", ctypes.c_int), ("exit_bc", ctypes.c_int), ("precision", ctypes.c_int),
                ("reorder", ctypes.c_int), ("cfl", ctypes.c_double), ("limiter_zeta", ctypes.c_double),
                ("limiter_zeta1", ctypes.c_double), ("inlet_rho", ctypes.c_double), ("inlet_p", ctypes.c_double),
                ("inlet_u", ctypes.c_double), ("inlet_v", ctypes.c_double), ("inlet_p0", ctypes.c_double),
                ("inlet_t0", ctypes.c_double), ("exit_p", ctypes.c_double), ("r_gas", ctypes.c_double),
                ("device", ctypes.c_int), ("stream", ctypes.c_void_p), ("weno", ctypes.c_int),
                ("weno_characteristic", ctypes.c_int), ("entropy_fix_linear", ctypes.c_double),
                ("shock_fix", ctypes.c_double), ("movers_single_alpha", ctypes.c_int),
                ("movers_entropy_fix", ctypes.c_int)]


class FluxArrays(ctypes.Structure):
    """cfd_flux_arrays: device pointers (integers) of one net-flux evaluation."""
    _fields_ = [("n_physical", ctypes.c_int), ("n_total", ctypes.c_int)] + \
               [(n, ctypes.c_void_p) for n in ("n_faces", "neighbours", "nx", "ny", "dl", "area", "inv_area",
                                                "second_neighbours", "d1", "d2", "degenerate", "prim", "U",
                                                "net_flux", "dt", "min_dt")]


class MlpSeg(ctypes.Structure):
    """cfd_mlp_seg: one input segment of a dense block (device pointers as integers)."""
    _fields_ = [("src", ctypes.c_void_p), ("idx", ctypes.c_void_p), ("width", ctypes.c_int), ("ld", ctypes.c_int),
                ("silu", ctypes.c_int)]


class MlpFwd(ctypes.Structure):
    """cfd_mlp_fwd."""
    _fields_ = [("rows", ctypes.c_int), ("nseg", ctypes.c_int), ("seg", MlpSeg * 3), ("out", ctypes.c_int),
                ("w1", ctypes.c_void_p), ("b1", ctypes.c_void_p), ("w2", ctypes.c_void_p), ("b2", ctypes.c_void_p),
                ("resid", ctypes.c_void_p), ("ld_resid", ctypes.c_int), ("z1", ctypes.c_void_p),
                ("y", ctypes.c_void_p), ("ld_y", ctypes.c_int), ("engine", ctypes.c_int)]


class MlpBwd(ctypes.Structure):
    """cfd_mlp_bwd."""
    _fields_ = [("rows", ctypes.c_int), ("in_width", ctypes.c_int), ("out", ctypes.c_int), ("dy", ctypes.c_void_p),
                ("ld_dy", ctypes.c_int), ("z1", ctypes.c_void_p), ("w1", ctypes.c_void_p), ("w2", ctypes.c_void_p),
                ("dz1", ctypes.c_void_p), ("dx", ctypes.c_void_p), ("ld_dx", ctypes.c_int), ("engine", ctypes.c_int)]


class MlpWgrad(ctypes.Structure):
    """cfd_mlp_wgrad."""
    _fields_ = [("rows", ctypes.c_int), ("n", ctypes.c_int), ("dz", ctypes.c_void_p), ("ld_dz", ctypes.c_int),
                ("nseg", ctypes.c_int), ("seg", MlpSeg * 3), ("workspace", ctypes.c_void_p), ("dw", ctypes.c_void_p),
                ("db", ctypes.c_void_p), ("accumulate", ctypes.c_int)]


class StepInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("min_dt", ctypes.c_double), ("total_time", ctypes.c_double),
                ("error", ctypes.c_double * 4), ("res_l2", ctypes.c_double * 4), ("bad_cell", ctypes.c_int),
                ("status", ctypes.c_int)]


# Every symbol include/cfd_b200.h declares, with its ctypes signature.
_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_DP = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "cfd_last_error": (ctypes.c_char_p, []),
    "cfd_version": (ctypes.c_char_p, []),
    "cfd_mesh_box": (_I, [_I, _I, _D, _D, _D, _D, ctypes.POINTER(_P)]),
    "cfd_mesh_half_cylinder": (_I, [_I, _I, _D, _D, _D, ctypes.POINTER(_P)]),
    "cfd_mesh_ramp": (_I, [_I, _I, _D, _D, _D, _D, _I, ctypes.POINTER(_P)]),
    "cfd_mesh_bump": (_I, [_I, _I, _D, _D, _D, _I, _D, ctypes.c_uint64, _I, ctypes.POINTER(_P)]),
    "cfd_mesh_read_vtk": (_I, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "cfd_mesh_write_vtk": (_I, [_P, ctypes.c_char_p]),
    "cfd_mesh_describe": (_I, [_P, ctypes.POINTER(MeshDesc)]),
    "cfd_mesh_centers": (_I, [_P, _DP]),
    "cfd_mesh_block_order": (_I, [ctypes.POINTER(MeshDesc), ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I),
                                  ctypes.POINTER(_I)]),
    "cfd_mesh_points": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_DP)]),
    "cfd_mesh_destroy": (None, [_P]),
    "cfd_config_default": (None, [ctypes.POINTER(Config)]),
    "cfd_config_read_json": (_I, [ctypes.c_char_p, ctypes.POINTER(Config)]),
    "cfd_create": (_I, [ctypes.POINTER(MeshDesc), ctypes.POINTER(Config), ctypes.POINTER(_P)]),
    "cfd_destroy": (None, [_P]),
    "cfd_upload_state": (_I, [_P, _DP, _I]),
    "cfd_step": (_I, [_P, _I, _D, ctypes.POINTER(StepInfo)]),
    "cfd_step_async": (_I, [_P, _I]),
    "cfd_sync": (_I, [_P, ctypes.POINTER(StepInfo)]),
    "cfd_set_option": (_I, [_P, ctypes.c_char_p, _D]),
    "cfd_autotune": (_I, [_P, _I, ctypes.c_char_p, ctypes.c_size_t]),
    "cfd_apply_boundary_conditions": (_I, [_P]),
    "cfd_evaluate_net_flux": (_I, [_P]),
    "cfd_lax_friedrichs": (_I, [_P]),
    "cfd_explicit_method": (_I, [_P]),
    "cfd_runge_kutta_method": (_I, [_P]),
    "cfd_estimate_error": (_I, [_P, _DP]),
    "cfd_update": (_I, [_P]),
    "cfd_get_min_dt": (_I, [_P, _DP]),
    "cfd_download": (_I, [_P, _DP, _DP, _DP, _DP, _DP]),
    "cfd_download_stage_state": (_I, [_P, _DP]),
    "cfd_download_U": (_I, [_P, _DP]),
    "cfd_upload_state_async": (_I, [_P, _DP, _I]),
    "cfd_download_U_async": (_I, [_P, _DP]),
    "cfd_gradient": (_I, [_P, _I, _DP]),
    "cfd_eval_limiter": (_I, [_I, _DP, _DP, _I, _DP, _I]),
    "cfd_write_solution": (_I, [_P, ctypes.c_char_p, ctypes.POINTER(_I), _I]),
    "cfd_read_solution": (_I, [_P, ctypes.c_char_p, _I]),
    "cfd_vtk_copy_grid": (_I, [ctypes.c_char_p, ctypes.c_char_p]),
    "cfd_vtk_append_solution": (_I, [ctypes.c_char_p, ctypes.c_char_p, _I]),
    "cfd_eval_face_flux": (_I, [_I, _I, _DP, _DP, _DP, _DP, _I, _DP, _I]),
    "cfd_amr_tags": (_I, [_P, _D, _D, _DP, ctypes.POINTER(ctypes.c_uint8)]),
    "cfd_kernel_time": (_I, [_P, ctypes.c_char_p, _DP, ctypes.POINTER(ctypes.c_longlong)]),
    "cfd_evaluate_net_flux_noalloc": (_I, [ctypes.POINTER(FluxArrays), ctypes.POINTER(Config), _P]),
    "cfd_face_count": (_I, [_P]),
    "cfd_batch_create": (_I, [_I, ctypes.POINTER(MeshDesc), _DP, ctypes.POINTER(Config), ctypes.POINTER(_P)]),
    "cfd_batch_upload_state": (_I, [_P, _DP]),
    "cfd_batch_download_state": (_I, [_P, _DP]),
    "cfd_batch_run": (_I, [_P, _I, _D, _I, ctypes.POINTER(_I), _DP, _DP, ctypes.POINTER(ctypes.c_longlong),
                           ctypes.POINTER(_I)]),
    "cfd_batch_destroy": (None, [_P]),
    "cfd_batch_set_boundary_values": (_I, [_P, _DP, _DP]),
    "cfd_set_delu": (_I, [_P, _DP]),
    "cfd_batch_set_option": (_I, [_P, ctypes.c_char_p, _D]),
    "cfd_mpnn_segment_sum": (_I, [_P, _P, _P, _I, _I, _P, _P]),
    "cfd_mpnn_mlp_forward": (_I, [ctypes.POINTER(MlpFwd), _P]),
    "cfd_mpnn_mlp_backward": (_I, [ctypes.POINTER(MlpBwd), _P]),
    "cfd_mpnn_weight_grad": (_I, [ctypes.POINTER(MlpWgrad), _P]),
    "cfd_mpnn_wgrad_blocks": (_I, []),
    "cfd_mpnn_status": (_I, [ctypes.POINTER(ctypes.c_int), _I]),
    "cfd_mpnn_add": (_I, [_P, _I, _P, _I, _P, _I, _I, _I, _P]),
    "cfd_mpnn_gather_add": (_I, [_P, _I, _P, _I, _P, _I, _I, _P]),
    "cfd_mpnn_segment_sum_acc": (_I, [_P, _I, _P, _P, _I, _I, _P, _I, _I, _P]),
    "cfd_mpnn_mse": (_I, [_P, _P, _I, _P, _P, _P]),
    "cfd_mpnn_adam": (_I, [_P, _P, _P, _P, _I, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _I,
                           _P]),
    "cfd_batch_set_reference_residual": (_I, [_P, _DP]),
    "cfd_batch_residuals": (_I, [_P, _DP]),
    "cfd_kernel_launches": (ctypes.c_longlong, [_P]),
    "cfd_device_bytes": (ctypes.c_size_t, [_P]),
}

_lib = None


def lib():
    """Loads libcfd_b200.so (building it first if the sources are newer and nvcc is present)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) or os.environ.get("CFD_B200_REBUILD"):
        from . import build as _build
        _build.build()
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(status):
    if status != CFD_OK:
        raise CfdError(status, lib().cfd_last_error().decode(errors="replace"))


def _dp(a):
    return a.ctypes.data_as(_DP)


class Mesh:
    """Host mesh in the reference layout (ghost ids cell-major/face-minor from NP)."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle) if not isinstance(handle, ctypes.c_void_p) else handle
        d = MeshDesc()
        _check(lib().cfd_mesh_describe(self._h, ctypes.byref(d)))
        self.desc = d
        self.n_physical = d.n_physical
        self.n_ghost = d.n_ghost
        self.n_total = d.n_physical + d.n_ghost
        NP = d.n_physical
        self.n_faces = np.ctypeslib.as_array(d.n_faces, (NP,)).copy()
        self.neighbours = np.ctypeslib.as_array(d.neighbours, (NP, 4)).copy()
        self.face_normals = np.ctypeslib.as_array(d.face_normals, (NP, 8)).copy()
        self.face_lengths = np.ctypeslib.as_array(d.face_lengths, (NP, 4)).copy()
        self.center_distances = np.ctypeslib.as_array(d.center_distances, (NP, 4)).copy()
        self.center_vectors = np.ctypeslib.as_array(d.center_vectors, (NP, 8)).copy()
        self.area = np.ctypeslib.as_array(d.area, (NP,)).copy()
        self.inv_area = np.ctypeslib.as_array(d.inv_area, (NP,)).copy()
        self.boundary = np.ctypeslib.as_array(d.boundary, (d.n_boundary, 4)).copy() if d.n_boundary else \
            np.zeros((0, 4), np.int32)
        c = np.zeros((self.n_total, 3))
        _check(lib().cfd_mesh_centers(self._h, _dp(c)))
        self.centers = c

    @classmethod
    def _make(cls, fn, *args):
        h = ctypes.c_void_p()
        _check(fn(*args, ctypes.byref(h)))
        return cls(h)

    @classmethod
    def box(cls, nx, ny, x0=0.0, x1=1.0, y0=0.0, y1=1.0):
        return cls._make(lib().cfd_mesh_box, nx, ny, x0, x1, y0, y1)

    @classmethod
    def half_cylinder(cls, ntheta, nr, r_body=1.0, r_outer=4.0, ratio=1.005):
        return cls._make(lib().cfd_mesh_half_cylinder, ntheta, nr, r_body, r_outer, ratio)

    @classmethod
    def ramp(cls, nx, ny, length=3.0, height=1.0, x_corner=1.0, angle_deg=15.0, open_top=False):
        return cls._make(lib().cfd_mesh_ramp, nx, ny, length, height, x_corner, angle_deg, 1 if open_top else 0)

    @classmethod
    def bump(cls, nx, ny, length=3.0, height=1.0, thickness=0.1, n_quad_layers=8, jitter=0.3, seed=1234,
             triangles=True):
        return cls._make(lib().cfd_mesh_bump, nx, ny, length, height, thickness, n_quad_layers, jitter, seed,
                         1 if triangles else 0)

    @classmethod
    def read_vtk(cls, path):
        return cls._make(lib().cfd_mesh_read_vtk, path.encode())

    def write_vtk(self, path):
        _check(lib().cfd_mesh_write_vtk(self._h, path.encode()))

    def block_order(self):
        """(ni, nj, lh, cells) of the structured-block numbering (reorder 4): cells[j * ni + i] is
        the mesh cell at (i, j).  Raises CfdError (CFD_ERR_MESH) when the mesh is not a single
        structured block of quads."""
        ni, nj, lh = _I(), _I(), _I()
        cells = np.zeros(self.n_physical, np.int32)
        _check(lib().cfd_mesh_block_order(ctypes.byref(self.desc), ctypes.byref(ni), ctypes.byref(nj), ctypes.byref(lh),
                                          cells.ctypes.data_as(ctypes.POINTER(_I))))
        return ni.value, nj.value, lh.value, cells

    def points(self):
        n = ctypes.c_int()
        p = _DP()
        _check(lib().cfd_mesh_points(self._h, ctypes.byref(n), ctypes.byref(p)))
        return np.ctypeslib.as_array(p, (n.value, 3)).copy()

    def __del__(self):
        try:
            if self._h:
                lib().cfd_mesh_destroy(self._h)
                self._h = None
        except Exception:
            pass


def default_config(**kw):
    c = Config()
    lib().cfd_config_default(ctypes.byref(c))
    for k, v in kw.items():
        if not hasattr(c, k):
            raise KeyError(k)
        setattr(c, k, v)
    return c


def read_config_json(path, **kw):
    c = default_config()
    _check(lib().cfd_config_read_json(path.encode(), ctypes.byref(c)))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


class Solver:
    """One device context over one mesh (the reference's solver globals, on the GPU)."""

    def __init__(self, mesh, config):
        self.mesh = mesh
        self.config = config
        h = ctypes.c_void_p()
        _check(lib().cfd_create(ctypes.byref(mesh.desc), ctypes.byref(config), ctypes.byref(h)))
        self._h = h
        self.info = StepInfo()
        self._pending = []  # host arrays of enqueued asynchronous copies, kept alive until sync()

    def close(self):
        if getattr(self, "_h", None):
            lib().cfd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state -----------------------------------------------------------------------------
    def upload_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        _check(lib().cfd_upload_state(self._h, _dp(U), U.shape[0]))

    def download(self):
        m = self.mesh
        U = np.zeros((m.n_total, 4))
        P = np.zeros((m.n_total, 11))
        dt = np.zeros(m.n_physical)
        net = np.zeros((m.n_physical, 4))
        dU = np.zeros((m.n_physical, 4))
        _check(lib().cfd_download(self._h, _dp(U), _dp(P), _dp(dt), _dp(net), _dp(dU)))
        return {"U": U, "prim": P, "dt": dt, "net_flux": net, "delU": dU}

    def download_U(self, out=None):
        if out is None:
            out = np.zeros((self.mesh.n_total, 4))
        _check(lib().cfd_download_U(self._h, _dp(out)))
        return out

    def stage_state(self):
        S = np.zeros((self.mesh.n_physical, 4))
        _check(lib().cfd_download_stage_state(self._h, _dp(S)))
        return S

    # -- reference entry points --------------------------------------------------------------
    def Apply_Boundary_Conditions(self):
        _check(lib().cfd_apply_boundary_conditions(self._h))

    def Evaluate_Cell_Net_Flux(self):
        _check(lib().cfd_evaluate_net_flux(self._h))

    def Explicit_Method(self):
        _check(lib().cfd_explicit_method(self._h))

    def Lax_Fedrichs(self):
        _check(lib().cfd_lax_friedrichs(self._h))

    def Runge_Kutta_Method(self):
        _check(lib().cfd_runge_kutta_method(self._h))

    def Estimate_Error(self):
        e = np.zeros(4)
        _check(lib().cfd_estimate_error(self._h, _dp(e)))
        return e

    def Update(self):
        _check(lib().cfd_update(self._h))

    def Set_DelU(self, dU):
        dU = np.ascontiguousarray(dU, np.float64)
        _check(lib().cfd_set_delu(self._h, dU.ctypes.data_as(_DP)))

    def get_Min_dt(self):
        v = ctypes.c_double()
        _check(lib().cfd_get_min_dt(self._h, ctypes.byref(v)))
        return v.value

    # -- whole steps ---------------------------------------------------------------------------
    def step(self, n=1, t_end=0.0):
        _check(lib().cfd_step(self._h, n, t_end, ctypes.byref(self.info)))
        return self.info

    def step_async(self, n):
        _check(lib().cfd_step_async(self._h, n))

    def upload_state_async(self, U):
        """Enqueues the upload of all NP+NG rows (cfd_upload_state_async) and returns; U (float64,
        C order, best page-locked) is kept alive until sync()."""
        if not (isinstance(U, np.ndarray) and U.dtype == np.float64 and U.flags.c_contiguous):
            raise ValueError("upload_state_async needs a C-contiguous float64 array")
        _check(lib().cfd_upload_state_async(self._h, _dp(U), U.shape[0]))
        self._pending.append(U)

    def download_U_async(self, out):
        """Enqueues the download of U_Cells into `out` ([NP+NG, 4] float64, best page-locked),
        which holds the result after sync()."""
        if not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous and
                out.size >= 4 * self.mesh.n_total):
            raise ValueError("download_U_async needs a C-contiguous float64 array of NP+NG rows")
        _check(lib().cfd_download_U_async(self._h, _dp(out)))
        self._pending.append(out)

    def sync(self):
        _check(lib().cfd_sync(self._h, ctypes.byref(self.info)))
        self._pending = []
        return self.info

    def write_solution(self, path, header=(0, 0, 0)):
        """Solution file in the reference's Write_Solution format (cfd_write_solution)."""
        h = (ctypes.c_int * len(header))(*header)
        _check(lib().cfd_write_solution(self._h, str(path).encode(), h, len(header)))

    def read_solution(self, path, n_header=3):
        """Restart from a solution file (cfd_read_solution)."""
        _check(lib().cfd_read_solution(self._h, str(path).encode(), n_header))

    def autotune(self, steps=20):
        """Picks the fastest bit-identical launch options on this mesh (cfd_autotune); returns
        the per-candidate report."""
        buf = ctypes.create_string_buffer(4096)
        _check(lib().cfd_autotune(self._h, steps, buf, len(buf)))
        return buf.value.decode()

    def set_option(self, name, value):
        _check(lib().cfd_set_option(self._h, name.encode(), float(value)))

    def gradient(self, var):
        g = np.zeros((self.mesh.n_physical, 2))
        _check(lib().cfd_gradient(self._h, var, _dp(g)))
        return g

    def amr_indicator(self):
        ind = np.zeros(self.mesh.n_physical)
        _check(lib().cfd_amr_tags(self._h, 0.0, 0.0, _dp(ind), ctypes.POINTER(ctypes.c_uint8)()))
        return ind

    def amr_tags(self, threshold, max_fraction):
        ind = np.zeros(self.mesh.n_physical)
        tags = np.zeros(self.mesh.n_physical, np.uint8)
        _check(lib().cfd_amr_tags(self._h, threshold, max_fraction, _dp(ind),
                                  tags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return ind, tags

    def kernel_time(self, kernel):
        """(total ms, launches) of a kernel family timed while option "profile" was set."""
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        _check(lib().cfd_kernel_time(self._h, kernel.encode(), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    @property
    def n_faces(self):
        return lib().cfd_face_count(self._h)

    @property
    def kernel_launches(self):
        return lib().cfd_kernel_launches(self._h)

    @property
    def device_bytes(self):
        return lib().cfd_device_bytes(self._h)


class Batch:
    """Many independent meshes solved together (cfd_batch_*)."""

    def __init__(self, meshes, config, inflow=None):
        self.meshes = list(meshes)
        n = len(self.meshes)
        descs = (MeshDesc * n)(*[m.desc for m in self.meshes])
        self._keep = descs
        infl = None
        if inflow is not None:
            self._inflow = np.ascontiguousarray(inflow, dtype=np.float64).reshape(n, 4)
            infl = _dp(self._inflow)
        h = ctypes.c_void_p()
        _check(lib().cfd_batch_create(n, descs, infl, ctypes.byref(config), ctypes.byref(h)))
        self._h = h
        self.rows = [m.n_total for m in self.meshes]

    def upload_state(self, states):
        U = np.ascontiguousarray(np.concatenate(states, axis=0), dtype=np.float64)
        _check(lib().cfd_batch_upload_state(self._h, _dp(U)))

    def set_boundary_values(self, inlet=None, exit_p=None):
        """Per-instance inlet values [n, 4] (read by the inlet kind) and exit pressures [n]."""
        n = len(self.meshes)
        self._bv = [None if inlet is None else np.ascontiguousarray(inlet, dtype=np.float64).reshape(n, 4),
                    None if exit_p is None else np.ascontiguousarray(exit_p, dtype=np.float64).reshape(n)]
        _check(lib().cfd_batch_set_boundary_values(self._h, None if self._bv[0] is None else _dp(self._bv[0]),
                                                   None if self._bv[1] is None else _dp(self._bv[1])))

    def set_reference_residual(self, r0=None):
        """Per-instance residual normalisers for run()'s tolerance (None: first-step residual)."""
        self._r0 = None if r0 is None else np.ascontiguousarray(r0, dtype=np.float64)
        _check(lib().cfd_batch_set_reference_residual(self._h, None if self._r0 is None else _dp(self._r0)))

    def residuals(self):
        """||R_rho||_2 of each instance's last residual evaluation."""
        r = np.zeros(len(self.meshes))
        _check(lib().cfd_batch_residuals(self._h, _dp(r)))
        return r

    def download_state(self):
        U = np.zeros((sum(self.rows), 4))
        _check(lib().cfd_batch_download_state(self._h, _dp(U)))
        out, r = [], 0
        for n in self.rows:
            out.append(U[r:r + n])
            r += n
        return out

    def set_option(self, name, value):
        _check(lib().cfd_batch_set_option(self._h, name.encode(), float(value)))

    def run(self, max_steps, tol, check_every=50):
        n = len(self.meshes)
        sto = (ctypes.c_int * n)()
        tto = np.zeros(n)
        rr = np.zeros(n)
        cu = ctypes.c_longlong()
        sd = ctypes.c_int()
        _check(lib().cfd_batch_run(self._h, max_steps, tol, check_every, sto, _dp(tto), _dp(rr), ctypes.byref(cu),
                                   ctypes.byref(sd)))
        return {"steps_to_tol": np.array(sto[:]), "time_to_tol": tto, "res_ratio": rr, "cell_updates": cu.value,
                "steps": sd.value}

    def close(self):
        if getattr(self, "_h", None):
            lib().cfd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def vtk_copy_grid(grid_vtk, out_vtk):
    """The grid part of a VTK file, copied as the reference's Read_Write_Grid does."""
    _check(lib().cfd_vtk_copy_grid(str(grid_vtk).encode(), str(out_vtk).encode()))


def vtk_append_solution(solution_txt, out_vtk, n_header=3):
    """Cell data of a solution file appended to a VTK file (the reference's Append_Solution)."""
    _check(lib().cfd_vtk_append_solution(str(solution_txt).encode(), str(out_vtk).encode(), n_header))


def eval_limiter(limiter, a, b, device=0):
    """phi(a, b) of the limiter family on the GPU (cfd_eval_limiter)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.zeros_like(a)
    _check(lib().cfd_eval_limiter(limiter, _dp(a), _dp(b), a.size, _dp(out), device))
    return out


def eval_face_flux(scheme, UL, UR, normals, lengths, precision=PREC_FP64, device=0):
    """Face fluxes [n, 4] of conserved left/right states [n, 4] on the GPU (cfd_eval_face_flux)."""
    UL = np.ascontiguousarray(UL, dtype=np.float64)
    UR = np.ascontiguousarray(UR, dtype=np.float64)
    normals = np.ascontiguousarray(normals, dtype=np.float64)
    lengths = np.ascontiguousarray(lengths, dtype=np.float64)
    n = UL.shape[0]
    F = np.zeros((n, 4))
    _check(lib().cfd_eval_face_flux(scheme, precision, _dp(UL), _dp(UR), _dp(normals), _dp(lengths), n, _dp(F),
                                    device))
    return F


def conserved_from_primitive(rho, u, v, p):
    """Calculate_Computational_Variables(P, V, Rho, 2) (src/Basic_Functions.cpp:249-283) per row."""
    rho = np.asarray(rho, np.float64)
    u = np.asarray(u, np.float64)
    v = np.asarray(v, np.float64)
    p = np.asarray(p, np.float64)
    vmag = 0.5 * (u * u + v * v)
    U = np.empty(rho.shape + (4,))
    U[..., 0] = rho
    U[..., 1] = rho * u
    U[..., 2] = rho * v
    U[..., 3] = (p / (1.4 - 1.0)) + rho * vmag
    return U
