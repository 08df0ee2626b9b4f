"""OverlappingBLs hot path on B200: Python binding of the C ABI (include/obl.h).

The product is libobl_b200.so (hand-written sm_100a CUDA kernels behind a C ABI).
This module loads it with ctypes and mirrors the reference's Fortran routine names
and argument order (output first, input second, as in ``call ddx(dfdx, fun)``,
SBL/code/004_derivatives.f90:18).  There is no CPU fallback: if the library is
missing or no GPU is present, constructing a Context raises.

Host arrays are numpy arrays in the reference's Fortran layout (``order='F'``):
    physical field  (ldx, nyt, nz+1)  float64     ldx = 2*(nxt/2+1), nz = nzt
    dpdx/dpdy/dpdz  (ldx, nyt, nz)    float64     (slot jz-1 holds level jz)
    padded field    (nxt2, nyt2, nlev)
    spectral        (lhx, nyt, nlev)  complex128
``*_dev`` methods take integer device pointers in the context's storage type
(float64 for precision="f64", float32 for "mixed"/"f32").
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# $OBL_LIB selects another build of the library (e.g. a tuning variant)
LIB_PATH = os.environ.get("OBL_LIB") or os.path.join(_HERE, "libobl_b200.so")

OBL_OK = 0
ERRORS = {1: "OBL_ERR_ARG", 2: "OBL_ERR_CUDA", 3: "OBL_ERR_NOMEM", 4: "OBL_ERR_TIMEOUT",
          5: "OBL_ERR_UNSUPPORTED", 6: "OBL_ERR_NODEV", 7: "OBL_ERR_IO"}
# the fields of a vel_tt restart file, in file order (012_io.f90:526-546)
VEL_TT_FIELDS = ("u", "v", "w", "RHSx", "RHSy", "RHSz", "Cs_opt2", "F_LM", "F_MM", "F_QN", "F_NN")
PRECISION = {"f64": 0, "mixed": 1, "f32": 2}
TOP_BC = {"single": 0, "neumann": 1}

# every symbol declared in include/obl.h
EXPORTS = [
    "obl_ctx_create", "obl_ctx_destroy", "obl_ctx_info", "obl_set_stream", "obl_synchronize",
    "obl_last_error", "obl_launch_count", "obl_timing_enable", "obl_timing_report",
    "obl_set_param", "obl_get_param",
    "obl_ddx", "obl_ddy", "obl_ddx_dev", "obl_ddy_dev",
    "obl_ddz_uv", "obl_ddz_w", "obl_ddz_uv_dev", "obl_ddz_w_dev",
    "obl_divstress_uv", "obl_divstress_w", "obl_divstress_uv_dev", "obl_divstress_w_dev",
    "obl_divstress_uv_slab_dev", "obl_divstress_w_slab_dev",
    "obl_write_file_3d_dev", "obl_read_file_3d_dev", "obl_checkpoint_final_dev", "obl_read_flow_field_dev",
    "obl_read_total_time", "obl_write_total_time", "obl_selftest_grid_barrier", "obl_check_report",
    "obl_check_selftest",
    "obl_fftn", "obl_ifftn", "obl_fftn_dev", "obl_ifftn_dev",
    "obl_zero_padding", "obl_zero_unpadding", "obl_zero_padding_dev", "obl_zero_unpadding_dev",
    "obl_zero_padding_noalloc_dev",
    "obl_filter_data", "obl_filter_data_dev",
    "obl_press_stag_array", "obl_press_stag_array_dev",
    "obl_dpdz", "obl_dpdz_dev", "obl_project", "obl_project_dev",
    "obl_step", "obl_step_f32", "obl_step_dev",
    "obl_convec", "obl_convec_dev", "obl_rollout_step", "obl_rollout_step_dev",
    "obl_rollout_step_vjp", "obl_rollout_step_vjp_dev", "obl_ke_band", "obl_ke_band_dev",
    "obl_rollout_grad", "obl_rollout_grad_dev",
    "obl_ensemble_create", "obl_ensemble_destroy", "obl_ensemble_size", "obl_ensemble_context",
    "obl_ensemble_set_mode", "obl_ensemble_get_mode", "obl_ensemble_step_dev",
    "obl_ensemble_capture_dev", "obl_ensemble_replay", "obl_ensemble_synchronize",
    "obl_ensemble_time_dev", "obl_ensemble_phase_times", "obl_ensemble_last_error",
    "obl_slab_sizes", "obl_slab_begin_dev", "obl_slab_solve_dev", "obl_slab_finish_dev",
]
ENS_MODES = {"sequential": 0, "concurrent": 1, "persistent": 2, "persistent_split": 3, "persistent_flow": 4}


class OblError(RuntimeError):
    pass


class Grid(ctypes.Structure):
    _fields_ = [("nxt", ctypes.c_int), ("nyt", ctypes.c_int), ("nzt", ctypes.c_int),
                ("lx_tot", ctypes.c_double), ("ly_tot", ctypes.c_double),
                ("lz_tot", ctypes.c_double), ("z_i", ctypes.c_double),
                ("dt", ctypes.c_double), ("u_scale", ctypes.c_double)]


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("top_bc", ctypes.c_int),
                ("ubc_stress_free", ctypes.c_int), ("fp64_k2_max", ctypes.c_double),
                ("device", ctypes.c_int)]


class Info(ctypes.Structure):
    _fields_ = [("nxt", ctypes.c_int), ("nyt", ctypes.c_int), ("nzt", ctypes.c_int),
                ("nz", ctypes.c_int), ("ldx", ctypes.c_int), ("lhx", ctypes.c_int),
                ("nxt2", ctypes.c_int), ("nyt2", ctypes.c_int), ("elem_bytes", ctypes.c_int),
                ("n_fp64_columns", ctypes.c_int), ("dz", ctypes.c_double),
                ("dt_nd", ctypes.c_double), ("lx", ctypes.c_double), ("ly", ctypes.c_double),
                ("field_elems", ctypes.c_longlong), ("dfield_elems", ctypes.c_longlong),
                ("big_elems", ctypes.c_longlong), ("spec_elems", ctypes.c_longlong)]


class StepIO(ctypes.Structure):
    _fields_ = [("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("w", ctypes.c_void_p),
                ("theta", ctypes.c_void_p), ("d", ctypes.c_void_p * 8),
                ("big", ctypes.c_void_p * 4), ("p", ctypes.c_void_p),
                ("dp", ctypes.c_void_p * 3), ("divtz_bot", ctypes.c_void_p),
                ("divtz_top", ctypes.c_void_p)]


_lib = None


def load_library(path=LIB_PATH):
    """Load libobl_b200.so; raises OblError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OblError(f"{path} is missing: build it with `python -m overlappingbls_b200.build`")
    L = ctypes.CDLL(path)
    P, I, C = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char)
    D, DP = ctypes.c_double, ctypes.POINTER(ctypes.c_double)
    ctx = ctypes.c_void_p
    sig = {
        "obl_ctx_create": [ctypes.POINTER(Grid), ctypes.POINTER(Options), ctypes.POINTER(ctypes.c_void_p)],
        "obl_ctx_destroy": [ctx], "obl_ctx_info": [ctx, ctypes.POINTER(Info)],
        "obl_set_stream": [ctx, P], "obl_synchronize": [ctx],
        "obl_last_error": [ctx, ctypes.c_char_p, ctypes.c_size_t],
        "obl_timing_enable": [ctx, I], "obl_timing_report": [ctx, ctypes.c_char_p, ctypes.c_size_t],
        "obl_set_param": [ctx, ctypes.c_char_p, ctypes.c_longlong],
        "obl_get_param": [ctx, ctypes.c_char_p, ctypes.POINTER(ctypes.c_longlong)],
        "obl_ddx": [ctx, P, P, I], "obl_ddy": [ctx, P, P, I],
        "obl_ddx_dev": [ctx, P, P, I], "obl_ddy_dev": [ctx, P, P, I],
        "obl_ddz_uv": [ctx, P, P], "obl_ddz_w": [ctx, P, P],
        "obl_ddz_uv_dev": [ctx, P, P], "obl_ddz_w_dev": [ctx, P, P],
        "obl_divstress_uv": [ctx, P, P, P, P], "obl_divstress_w": [ctx, P, P, P, P],
        "obl_divstress_uv_dev": [ctx, P, P, P, P], "obl_divstress_w_dev": [ctx, P, P, P, P],
        "obl_divstress_uv_slab_dev": [ctx, P, P, P, P, I, I], "obl_divstress_w_slab_dev": [ctx, P, P, P, P, I, I],
        "obl_write_file_3d_dev": [ctx, P, ctypes.c_char_p, ctypes.c_longlong, I, I],
        "obl_read_file_3d_dev": [ctx, P, ctypes.c_char_p, ctypes.c_longlong, I, I],
        "obl_checkpoint_final_dev": [ctx, ctypes.c_char_p, I, ctypes.POINTER(P), I, I],
        "obl_read_flow_field_dev": [ctx, ctypes.c_char_p, I, ctypes.POINTER(P), I, I],
        "obl_read_total_time": [ctypes.c_char_p, ctypes.POINTER(I)],
        "obl_write_total_time": [ctypes.c_char_p, I],
        "obl_selftest_grid_barrier": [ctx, I],
        "obl_check_report": [ctypes.POINTER(ctypes.c_longlong), ctypes.c_char_p, ctypes.c_size_t],
        "obl_check_selftest": [],
        "obl_fftn": [ctx, P, P, I], "obl_ifftn": [ctx, P, P, I],
        "obl_fftn_dev": [ctx, P, P, I], "obl_ifftn_dev": [ctx, P, P, I],
        "obl_zero_padding": [ctx, P, P, I], "obl_zero_unpadding": [ctx, P, P, I],
        "obl_zero_padding_dev": [ctx, P, P, I], "obl_zero_unpadding_dev": [ctx, P, P, I],
        "obl_zero_padding_noalloc_dev": [ctx, P, P, I],
        "obl_filter_data": [ctx, P, I], "obl_filter_data_dev": [ctx, P, I],
        "obl_press_stag_array": [ctx, P, P, P, P, P, P, P, P],
        "obl_press_stag_array_dev": [ctx, P, P, P, P, P, P, P, P],
        "obl_dpdz": [ctx, P, P], "obl_dpdz_dev": [ctx, P, P],
        "obl_project": [ctx, P, P, P, P, P, P], "obl_project_dev": [ctx, P, P, P, P, P, P],
        "obl_step": [ctx, ctypes.POINTER(StepIO)], "obl_step_f32": [ctx, ctypes.POINTER(StepIO)],
        "obl_step_dev": [ctx, ctypes.POINTER(StepIO)],
        "obl_convec": [ctx, P, P, P, P, P, P], "obl_convec_dev": [ctx, P, P, P, P, P, P],
        "obl_rollout_step": [ctx, P, P, P], "obl_rollout_step_dev": [ctx, P, P, P],
        "obl_rollout_step_vjp": [ctx, P, P, P, P, P, P],
        "obl_rollout_step_vjp_dev": [ctx, P, P, P, P, P, P],
        "obl_ke_band": [ctx, P, P, P, D, D, DP, P, P, P],
        "obl_ke_band_dev": [ctx, P, P, P, D, D, DP, P, P, P],
        "obl_rollout_grad": [ctx, I, P, P, P, D, D, DP, P, P, P],
        "obl_rollout_grad_dev": [ctx, I, P, P, P, D, D, DP, P, P, P],
    }
    E, IP = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)
    sig.update({
        "obl_ensemble_create": [ctypes.POINTER(Grid), I, ctypes.POINTER(Options), ctypes.POINTER(ctypes.c_void_p)],
        "obl_ensemble_destroy": [E], "obl_ensemble_size": [E],
        "obl_ensemble_context": [E, I, ctypes.POINTER(ctypes.c_void_p)],
        "obl_ensemble_set_mode": [E, I, I], "obl_ensemble_get_mode": [E, IP, IP, IP],
        "obl_ensemble_step_dev": [E, ctypes.POINTER(StepIO)],
        "obl_ensemble_capture_dev": [E, ctypes.POINTER(StepIO)], "obl_ensemble_replay": [E],
        "obl_ensemble_synchronize": [E],
        "obl_ensemble_time_dev": [E, ctypes.POINTER(StepIO), I, I, I, DP],
        "obl_ensemble_phase_times": [E, I, DP, I],
        "obl_slab_sizes": [ctx, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)],
        "obl_slab_begin_dev": [ctx, ctypes.POINTER(StepIO), I, I, P],
        "obl_slab_solve_dev": [ctx, P, I, I, P],
        "obl_slab_finish_dev": [ctx, ctypes.POINTER(StepIO), P, I, I],
        "obl_ensemble_last_error": [E, ctypes.c_char_p, ctypes.c_size_t],
    })
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = I
    L.obl_launch_count.argtypes = [ctx]
    L.obl_launch_count.restype = ctypes.c_longlong
    _lib = L
    return L


def _ptr(a, dtype=np.float64):
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if not isinstance(a, np.ndarray):
        raise TypeError("expected a numpy array or an integer device pointer")
    if a.dtype != dtype:
        raise TypeError(f"expected dtype {np.dtype(dtype)}, got {a.dtype}")
    if not (a.flags["F_CONTIGUOUS"] or a.ndim <= 1):
        raise TypeError("host arrays must be Fortran-ordered (order='F')")
    return a.ctypes.data


class Context:
    """One grid on one GPU: replaces init_parameter / init_fft_plan / init_coef_press."""

    def __init__(self, nxt, nyt, nzt, lx_tot, ly_tot, lz_tot, z_i, dt, u_scale=1.0,
                 precision="f64", top_bc="neumann", ubc_stress_free=False, fp64_k2_max=-1.0,
                 device=0):
        self._lib = load_library()
        g = Grid(nxt, nyt, nzt, lx_tot, ly_tot, lz_tot, z_i, dt, u_scale)
        o = Options(PRECISION[precision], TOP_BC[top_bc], 1 if ubc_stress_free else 0,
                    float(fp64_k2_max), int(device))
        h = ctypes.c_void_p()
        rc = self._lib.obl_ctx_create(ctypes.byref(g), ctypes.byref(o), ctypes.byref(h))
        if rc != OBL_OK:
            raise OblError(f"obl_ctx_create failed: {ERRORS.get(rc, rc)}")
        self._h = h
        self.precision = precision
        self.top_bc = top_bc
        inf = Info()
        self._lib.obl_ctx_info(self._h, ctypes.byref(inf))
        self.info = {k: getattr(inf, k) for k, _ in Info._fields_}
        for k in ("nxt", "nyt", "nzt", "nz", "ldx", "lhx", "nxt2", "nyt2", "dz", "dt_nd"):
            setattr(self, k, self.info[k])
        self.dtype = np.float64 if self.info["elem_bytes"] == 8 else np.float32

    @classmethod
    def _borrow(cls, handle, precision):
        """A non-owning view of a context that another object (an Ensemble) owns."""
        self = cls.__new__(cls)
        self._lib = load_library()
        self._h = ctypes.c_void_p(handle)
        self._owned = False
        self.precision = precision
        inf = Info()
        self._lib.obl_ctx_info(self._h, ctypes.byref(inf))
        self.info = {k: getattr(inf, k) for k, _ in Info._fields_}
        for k in ("nxt", "nyt", "nzt", "nz", "ldx", "lhx", "nxt2", "nyt2", "dz", "dt_nd"):
            setattr(self, k, self.info[k])
        self.dtype = np.float64 if self.info["elem_bytes"] == 8 else np.float32
        return self

    # ---- lifecycle / plumbing ----
    def close(self):
        if getattr(self, "_h", None) and getattr(self, "_owned", True):
            self._lib.obl_ctx_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc != OBL_OK:
            buf = ctypes.create_string_buffer(1024)
            self._lib.obl_last_error(self._h, buf, 1024)
            raise OblError(f"{what}: {ERRORS.get(rc, rc)} {buf.value.decode()}")

    def set_stream(self, stream_handle):
        self._check(self._lib.obl_set_stream(self._h, stream_handle), "obl_set_stream")

    def synchronize(self):
        self._check(self._lib.obl_synchronize(self._h), "obl_synchronize")

    def launch_count(self):
        return int(self._lib.obl_launch_count(self._h))

    def set_param(self, name, value):
        self._check(self._lib.obl_set_param(self._h, name.encode(), int(value)), "obl_set_param")

    def get_param(self, name):
        v = ctypes.c_longlong()
        self._check(self._lib.obl_get_param(self._h, name.encode(), ctypes.byref(v)), "obl_get_param")
        return v.value

    def timing(self, on=True):
        self._check(self._lib.obl_timing_enable(self._h, 1 if on else 0), "obl_timing_enable")

    def timing_report(self):
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(self._lib.obl_timing_report(self._h, buf, 1 << 16), "obl_timing_report")
        return json.loads(buf.value.decode())

    # ---- array helpers (Fortran layout) ----
    def field(self, nlev=None, dtype=np.float64):
        return np.zeros((self.ldx, self.nyt, self.nz + 1 if nlev is None else nlev), dtype, order="F")

    def dfield(self, dtype=np.float64):
        return np.zeros((self.ldx, self.nyt, self.nz), dtype, order="F")

    def big_field(self, nlev=None, dtype=np.float64):
        return np.zeros((self.nxt2, self.nyt2, self.nz + 1 if nlev is None else nlev), dtype, order="F")

    def spectral(self, nlev=None):
        return np.zeros((self.lhx, self.nyt, self.nz + 1 if nlev is None else nlev), np.complex128,
                        order="F")

    @staticmethod
    def _nlev(a):
        return a.shape[2] if a.ndim == 3 else 1

    # ---- reference routines, host arrays (output first, as in the Fortran) ----
    def ddx(self, dfdx, fun):
        self._check(self._lib.obl_ddx(self._h, _ptr(dfdx), _ptr(fun), self._nlev(fun)), "ddx")

    def ddy(self, dfdy, fun):
        self._check(self._lib.obl_ddy(self._h, _ptr(dfdy), _ptr(fun), self._nlev(fun)), "ddy")

    def ddz_uv(self, dfdz, fun):
        self._check(self._lib.obl_ddz_uv(self._h, _ptr(dfdz), _ptr(fun)), "ddz_uv")

    def ddz_w(self, dfdz, fun):
        self._check(self._lib.obl_ddz_w(self._h, _ptr(dfdz), _ptr(fun)), "ddz_w")

    def divstress_uv(self, divt, tx, ty, tz):
        """divt = div of the stress row (tx, ty, tz) at uv nodes (107_divstress.f90:4-44)."""
        self._check(self._lib.obl_divstress_uv(self._h, _ptr(divt), _ptr(tx), _ptr(ty), _ptr(tz)),
                    "divstress_uv")

    def divstress_w(self, divt, tx, ty, tz):
        """divt = div of the stress row (tx, ty, tz) at w nodes (107_divstress.f90:48-104)."""
        self._check(self._lib.obl_divstress_w(self._h, _ptr(divt), _ptr(tx), _ptr(ty), _ptr(tz)),
                    "divstress_w")

    def fftn(self, fin, fout):
        self._check(self._lib.obl_fftn(self._h, _ptr(fin), _ptr(fout, np.complex128),
                                       self._nlev(fin)), "fftn")

    def ifftn(self, fin, fout):
        self._check(self._lib.obl_ifftn(self._h, _ptr(fin, np.complex128), _ptr(fout),
                                        self._nlev(fout)), "ifftn")

    def zero_padding(self, var, var_big):
        self._check(self._lib.obl_zero_padding(self._h, _ptr(var), _ptr(var_big),
                                               self._nlev(var)), "zero_padding")

    def zero_unpadding(self, var_big, var):
        self._check(self._lib.obl_zero_unpadding(self._h, _ptr(var_big), _ptr(var),
                                                 self._nlev(var_big)), "zero_unpadding")

    def filter_data(self, f):
        self._check(self._lib.obl_filter_data(self._h, _ptr(f), self._nlev(f)), "filter_data")

    def press_stag_array(self, func, dfdx, dfdy, u, v, w, divtz_bot=None, divtz_top=None):
        self._check(self._lib.obl_press_stag_array(
            self._h, _ptr(u), _ptr(v), _ptr(w), _ptr(divtz_bot), _ptr(divtz_top),
            _ptr(func), _ptr(dfdx), _ptr(dfdy)), "press_stag_array")

    def dpdz(self, dpdz, p):
        self._check(self._lib.obl_dpdz(self._h, _ptr(p), _ptr(dpdz)), "dpdz")

    def project(self, u, v, w, dpdx, dpdy, dpdz):
        self._check(self._lib.obl_project(self._h, _ptr(u), _ptr(v), _ptr(w), _ptr(dpdx),
                                          _ptr(dpdy), _ptr(dpdz)), "project")

    def _stepio(self, u, v, w, theta, d, big, p, dp, divtz_bot=None, divtz_top=None, dtype=np.float64):
        io = StepIO()
        pp = lambda a: _ptr(a, dtype)
        io.u, io.v, io.w, io.theta, io.p = pp(u), pp(v), pp(w), pp(theta), pp(p)
        for i in range(8):
            io.d[i] = pp(d[i])
        for i in range(4):
            io.big[i] = pp(big[i])
        for i in range(3):
            io.dp[i] = pp(dp[i])
        io.divtz_bot, io.divtz_top = pp(divtz_bot), pp(divtz_top)
        return io

    def step(self, u, v, w, theta, d, big, p, dp, divtz_bot=None, divtz_top=None):
        """Fused step with host arrays (float64, or float32 through obl_step_f32)."""
        dt = u.dtype.type if isinstance(u, np.ndarray) else np.float64
        io = self._stepio(u, v, w, theta, d, big, p, dp, divtz_bot, divtz_top, dt)
        fn = self._lib.obl_step_f32 if dt == np.float32 else self._lib.obl_step
        self._check(fn(self._h, ctypes.byref(io)), "step")

    # ---- device-pointer variants (integers; storage type) ----
    def ddx_dev(self, dfdx, fun, nlev):
        self._check(self._lib.obl_ddx_dev(self._h, dfdx, fun, nlev), "ddx_dev")

    def ddy_dev(self, dfdy, fun, nlev):
        self._check(self._lib.obl_ddy_dev(self._h, dfdy, fun, nlev), "ddy_dev")

    def ddz_uv_dev(self, dfdz, fun):
        self._check(self._lib.obl_ddz_uv_dev(self._h, dfdz, fun), "ddz_uv_dev")

    def ddz_w_dev(self, dfdz, fun):
        self._check(self._lib.obl_ddz_w_dev(self._h, dfdz, fun), "ddz_w_dev")

    def selftest_grid_barrier(self, never_released=False):
        """The persistent ensemble kernel's grid barrier in one CTA: returns when it
        releases; raises OblError (OBL_ERR_TIMEOUT) when its bounded wait gives up."""
        self._check(self._lib.obl_selftest_grid_barrier(self._h, 1 if never_released else 0),
                    "selftest_grid_barrier")

    # ---- restart files (integer device pointers; FP64 files, see include/obl.h) ----
    def write_file_3d_dev(self, var, fn, disp0=0, zrank=0, nzranks=1):
        """write_file_mpi_3d (202_parallel.f90:1084-1120): levels 1..nz-1 of var."""
        self._check(self._lib.obl_write_file_3d_dev(self._h, var, os.fsencode(fn), disp0, zrank, nzranks),
                    "write_file_3d_dev")

    def read_file_3d_dev(self, var, fn, disp0=0, zrank=0, nzranks=1):
        """read_file_mpi_3d (202_parallel.f90:1211-1250): levels 1..nz-1 of var."""
        self._check(self._lib.obl_read_file_3d_dev(self._h, var, os.fsencode(fn), disp0, zrank, nzranks),
                    "read_file_3d_dev")

    @staticmethod
    def _vel_tt_ptrs(fields):
        if isinstance(fields, dict):
            fields = [fields.get(k) for k in VEL_TT_FIELDS]
        fields = list(fields)
        if len(fields) != len(VEL_TT_FIELDS):
            raise ValueError(f"vel_tt holds {len(VEL_TT_FIELDS)} fields {VEL_TT_FIELDS}")
        return (ctypes.c_void_p * len(fields))(*[f if f else None for f in fields])

    def checkpoint_final_dev(self, path_restart, nums, fields, zrank=0, nzranks=1):
        """checkpoint_final (012_io.f90:496-546): vel_tt%08d.out from device fields (a list
        in VEL_TT_FIELDS order or a dict by name; missing fields are written as zeros)."""
        self._check(self._lib.obl_checkpoint_final_dev(self._h, os.fsencode(path_restart), nums,
                                                       self._vel_tt_ptrs(fields), zrank, nzranks),
                    "checkpoint_final_dev")

    def read_flow_field_dev(self, path_restart, nums, fields, zrank=0, nzranks=1):
        """read_flow_field (102_01_ic.f90:682-734) into device fields (missing ones skipped)."""
        self._check(self._lib.obl_read_flow_field_dev(self._h, os.fsencode(path_restart), nums,
                                                      self._vel_tt_ptrs(fields), zrank, nzranks),
                    "read_flow_field_dev")

    def divstress_uv_dev(self, divt, tx, ty, tz):
        self._check(self._lib.obl_divstress_uv_dev(self._h, divt, tx, ty, tz), "divstress_uv_dev")

    def divstress_w_dev(self, divt, tx, ty, tz):
        self._check(self._lib.obl_divstress_w_dev(self._h, divt, tx, ty, tz), "divstress_w_dev")

    def divstress_uv_slab_dev(self, divt, tx, ty, tz, rank, nranks):
        self._check(self._lib.obl_divstress_uv_slab_dev(self._h, divt, tx, ty, tz, rank, nranks),
                    "divstress_uv_slab_dev")

    def divstress_w_slab_dev(self, divt, tx, ty, tz, rank, nranks):
        self._check(self._lib.obl_divstress_w_slab_dev(self._h, divt, tx, ty, tz, rank, nranks),
                    "divstress_w_slab_dev")

    def zero_padding_dev(self, var, var_big, nlev):
        self._check(self._lib.obl_zero_padding_dev(self._h, var, var_big, nlev), "zero_padding_dev")

    def zero_padding_noalloc_dev(self, var, var_big, nlev):
        """zero_padding through a static device scratch, allocating nothing: for callers
        that cannot allocate device memory when they call (an application whose memory
        pool owns all device memory after start-up, or a latency-critical path where
        cudaMalloc may block).  Limits as obl.h states (OBL_NOALLOC_SCRATCH_BYTES)."""
        self._check(self._lib.obl_zero_padding_noalloc_dev(self._h, var, var_big, nlev),
                    "zero_padding_noalloc_dev")

    def zero_unpadding_dev(self, var_big, var, nlev):
        self._check(self._lib.obl_zero_unpadding_dev(self._h, var_big, var, nlev), "zero_unpadding_dev")

    def fftn_dev(self, fin, fout, nlev):
        self._check(self._lib.obl_fftn_dev(self._h, fin, fout, nlev), "fftn_dev")

    def ifftn_dev(self, fin, fout, nlev):
        self._check(self._lib.obl_ifftn_dev(self._h, fin, fout, nlev), "ifftn_dev")

    def filter_data_dev(self, f, nlev):
        self._check(self._lib.obl_filter_data_dev(self._h, f, nlev), "filter_data_dev")

    def press_stag_array_dev(self, func, dfdx, dfdy, u, v, w, divtz_bot=None, divtz_top=None):
        self._check(self._lib.obl_press_stag_array_dev(self._h, u, v, w, divtz_bot, divtz_top,
                                                       func, dfdx, dfdy), "press_stag_array_dev")

    def dpdz_dev(self, dpdz, p):
        self._check(self._lib.obl_dpdz_dev(self._h, p, dpdz), "dpdz_dev")

    def project_dev(self, u, v, w, dpdx, dpdy, dpdz):
        self._check(self._lib.obl_project_dev(self._h, u, v, w, dpdx, dpdy, dpdz), "project_dev")

    def step_dev(self, u, v, w, theta, d, big, p, dp, divtz_bot=None, divtz_top=None):
        io = StepIO()
        io.u, io.v, io.w, io.theta, io.p = u, v, w, theta, p
        for i in range(8):
            io.d[i] = d[i]
        for i in range(4):
            io.big[i] = big[i]
        for i in range(3):
            io.dp[i] = dp[i]
        io.divtz_bot, io.divtz_top = divtz_bot, divtz_top
        self._check(self._lib.obl_step_dev(self._h, ctypes.byref(io)), "step_dev")

    # ---- z-slab of a split domain (device pointers; see overlappingbls_b200/slab.py) ----
    def slab_sizes(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self._lib.obl_slab_sizes(self._h, ctypes.byref(a), ctypes.byref(b)), "obl_slab_sizes")
        return a.value, b.value

    def slab_begin_dev(self, io, rank, nranks, plane_out):
        self._check(self._lib.obl_slab_begin_dev(self._h, ctypes.byref(io), int(rank), int(nranks), plane_out),
                    "obl_slab_begin_dev")

    def slab_solve_dev(self, plane_above, rank, nranks, iface_out):
        self._check(self._lib.obl_slab_solve_dev(self._h, plane_above, int(rank), int(nranks), iface_out),
                    "obl_slab_solve_dev")

    def slab_finish_dev(self, io, iface_all, rank, nranks):
        self._check(self._lib.obl_slab_finish_dev(self._h, ctypes.byref(io), iface_all, int(rank), int(nranks)),
                    "obl_slab_finish_dev")

    # ---- rollout problem of the adjoint (host arrays, float64) ----
    def convec(self, cx, cy, cz, u, v, w):
        """convec(cx, cy, cz) of 108_convec.f90 at the state u, v, w (levels 1..nz-1)."""
        self._check(self._lib.obl_convec(self._h, _ptr(u), _ptr(v), _ptr(w), _ptr(cx), _ptr(cy),
                                         _ptr(cz)), "convec")

    def rollout_step(self, u, v, w):
        """u1 = P(u - dt*tadv1*convec(u)), in place."""
        self._check(self._lib.obl_rollout_step(self._h, _ptr(u), _ptr(v), _ptr(w)), "rollout_step")

    def rollout_step_vjp(self, u, v, w, lu, lv, lw):
        """lu, lv, lw <- (d step / d state)^T (lu, lv, lw) at the state u, v, w, in place."""
        self._check(self._lib.obl_rollout_step_vjp(self._h, _ptr(u), _ptr(v), _ptr(w), _ptr(lu),
                                                   _ptr(lv), _ptr(lw)), "rollout_step_vjp")

    def ke_band(self, u, v, w, z_lo, z_hi, lu=None, lv=None, lw=None):
        J = ctypes.c_double(0.0)
        self._check(self._lib.obl_ke_band(self._h, _ptr(u), _ptr(v), _ptr(w), float(z_lo),
                                          float(z_hi), ctypes.byref(J), _ptr(lu), _ptr(lv),
                                          _ptr(lw)), "ke_band")
        return J.value

    def rollout_grad(self, nsteps, u0, v0, w0, z_lo, z_hi, gu=None, gv=None, gw=None):
        """J of the state after nsteps rollout steps; gu, gv, gw (optional outputs)
        receive dJ/d(u0, v0, w0)."""
        J = ctypes.c_double(0.0)
        self._check(self._lib.obl_rollout_grad(self._h, int(nsteps), _ptr(u0), _ptr(v0), _ptr(w0),
                                               float(z_lo), float(z_hi), ctypes.byref(J), _ptr(gu),
                                               _ptr(gv), _ptr(gw)), "rollout_grad")
        return J.value

    # ---- the same on device pointers (storage type) ----
    def convec_dev(self, cx, cy, cz, u, v, w):
        self._check(self._lib.obl_convec_dev(self._h, u, v, w, cx, cy, cz), "convec_dev")

    def rollout_step_dev(self, u, v, w):
        self._check(self._lib.obl_rollout_step_dev(self._h, u, v, w), "rollout_step_dev")

    def rollout_step_vjp_dev(self, u, v, w, lu, lv, lw):
        self._check(self._lib.obl_rollout_step_vjp_dev(self._h, u, v, w, lu, lv, lw),
                    "rollout_step_vjp_dev")

    def ke_band_dev(self, u, v, w, z_lo, z_hi, lu=None, lv=None, lw=None):
        J = ctypes.c_double(0.0)
        self._check(self._lib.obl_ke_band_dev(self._h, u, v, w, float(z_lo), float(z_hi),
                                              ctypes.byref(J), lu, lv, lw), "ke_band_dev")
        return J.value

    def rollout_grad_dev(self, nsteps, u0, v0, w0, z_lo, z_hi, gu=None, gv=None, gw=None):
        J = ctypes.c_double(0.0)
        self._check(self._lib.obl_rollout_grad_dev(self._h, int(nsteps), u0, v0, w0, float(z_lo),
                                                   float(z_hi), ctypes.byref(J), gu, gv, gw),
                    "rollout_grad_dev")
        return J.value


def read_total_time(fn):
    """The step number of total_time.dat (0 when the file is missing, as the reference)."""
    L = load_library()
    n = ctypes.c_int(0)
    rc = L.obl_read_total_time(os.fsencode(fn), ctypes.byref(n))
    if rc:
        raise OblError(f"read_total_time({fn}): {ERRORS.get(rc, rc)}")
    return n.value


def check_report():
    """(failed index checks since the last call, description of the first) of the
    bounds-checked build (-DOBL_CHECK=1); (-1, "") with the product build."""
    n = ctypes.c_longlong(0)
    buf = ctypes.create_string_buffer(256)
    rc = load_library().obl_check_report(ctypes.byref(n), buf, 256)
    if rc:
        raise OblError(f"check_report: {ERRORS.get(rc, rc)}")
    return n.value, buf.value.decode()


def check_selftest():
    """Bounds-checked build: record one failed check (no access made); see check_report."""
    rc = load_library().obl_check_selftest()
    if rc:
        raise OblError(f"check_selftest: {ERRORS.get(rc, rc)}")


def write_total_time(fn, nums):
    """total_time.dat as the reference writes it (one list-directed integer)."""
    rc = load_library().obl_write_total_time(os.fsencode(fn), int(nums))
    if rc:
        raise OblError(f"write_total_time({fn}): {ERRORS.get(rc, rc)}")


def stepio_dev(u, v, w, theta, d, big, p, dp, divtz_bot=None, divtz_top=None):
    """obl_step_io of integer device pointers."""
    io = StepIO()
    io.u, io.v, io.w, io.theta, io.p = u, v, w, theta, p
    for i in range(8):
        io.d[i] = d[i]
    for i in range(4):
        io.big[i] = big[i]
    for i in range(3):
        io.dp[i] = dp[i]
    io.divtz_bot, io.divtz_top = divtz_bot, divtz_top
    return io


class Ensemble:
    """Many independent instances (one grid each) advanced through obl_step together.

    grids: list of dicts with nxt, nyt, nzt, lx_tot, ly_tot, lz_tot, z_i, dt (u_scale)."""

    def __init__(self, grids, precision="mixed", top_bc="neumann", ubc_stress_free=False,
                 fp64_k2_max=-1.0, device=0):
        self._lib = load_library()
        n = len(grids)
        G = (Grid * n)()
        for i, g in enumerate(grids):
            G[i] = Grid(g["nxt"], g["nyt"], g["nzt"], g["lx_tot"], g["ly_tot"], g["lz_tot"], g["z_i"],
                        g["dt"], g.get("u_scale", 1.0))
        o = Options(PRECISION[precision], TOP_BC[top_bc], 1 if ubc_stress_free else 0,
                    float(fp64_k2_max), int(device))
        h = ctypes.c_void_p()
        rc = self._lib.obl_ensemble_create(G, n, ctypes.byref(o), ctypes.byref(h))
        if rc != OBL_OK:
            raise OblError(f"obl_ensemble_create failed: {ERRORS.get(rc, rc)}")
        self._h = h
        self.n = n
        self.precision = precision
        self.contexts = []
        for i in range(n):
            c = ctypes.c_void_p()
            self._check(self._lib.obl_ensemble_context(self._h, i, ctypes.byref(c)), "obl_ensemble_context")
            self.contexts.append(Context._borrow(c.value, precision))

    def close(self):
        if getattr(self, "_h", None):
            for c in self.contexts:
                c._h = None
            self._lib.obl_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != OBL_OK:
            buf = ctypes.create_string_buffer(1024)
            self._lib.obl_ensemble_last_error(self._h, buf, 1024)
            raise OblError(f"{what}: {ERRORS.get(rc, rc)} {buf.value.decode()}")

    def _ios(self, ios):
        if len(ios) != self.n:
            raise ValueError(f"expected {self.n} step buffers, got {len(ios)}")
        arr = (StepIO * self.n)()
        for i, io in enumerate(ios):
            arr[i] = io
        return arr

    def set_mode(self, mode, blocks_per_sm=0):
        self._check(self._lib.obl_ensemble_set_mode(self._h, ENS_MODES[mode], int(blocks_per_sm)),
                    "obl_ensemble_set_mode")

    def get_mode(self):
        m, b, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.obl_ensemble_get_mode(self._h, ctypes.byref(m), ctypes.byref(b),
                                                    ctypes.byref(nb)), "obl_ensemble_get_mode")
        name = {v: k for k, v in ENS_MODES.items()}[m.value]
        return name, b.value, nb.value

    def step_dev(self, ios):
        self._check(self._lib.obl_ensemble_step_dev(self._h, self._ios(ios)), "obl_ensemble_step_dev")

    def capture_dev(self, ios):
        self._check(self._lib.obl_ensemble_capture_dev(self._h, self._ios(ios)), "obl_ensemble_capture_dev")

    def replay(self):
        self._check(self._lib.obl_ensemble_replay(self._h), "obl_ensemble_replay")

    def synchronize(self):
        self._check(self._lib.obl_ensemble_synchronize(self._h), "obl_ensemble_synchronize")

    def time_dev(self, ios, use_graph=True, warmup=3, reps=10):
        ms = ctypes.c_double(0.0)
        self._check(self._lib.obl_ensemble_time_dev(self._h, self._ios(ios), 1 if use_graph else 0,
                                                    int(warmup), int(reps), ctypes.byref(ms)),
                    "obl_ensemble_time_dev")
        return ms.value

    def phase_times(self, on=True):
        """Turn the persistent kernel's phase stamps on/off; returns the 6 phase times (ms)
        of the last persistent step."""
        ms = (ctypes.c_double * 6)()
        self._check(self._lib.obl_ensemble_phase_times(self._h, 1 if on else 0, ms, 6),
                    "obl_ensemble_phase_times")
        return list(ms)
