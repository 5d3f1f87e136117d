"""Python binding of libsph_b200 (ctypes over the C-ABI in include/sph_b200.h).

This module is the host-side mirror of the reference's Fortran driver for the
weakly-compressible SPH step of SPH-2D:

  * ``SphConfig`` is the ``sph_config`` struct, filled the way the Fortran shim
    fills it from ``information_module`` (Taylor_Green_Vortex/information_module.f90).
  * ``Simulation.find_particle_pair`` / ``single_step_compute`` / ``time_iteration``
    mirror ``find_particle_pair()`` (Taylor_Green_Vortex/find_particle_pair.f90:21),
    ``single_step_compute()`` (Taylor_Green_Vortex/single_step_compute.f90:19) and the
    Runge-Kutta branch of ``time_iteration()`` (Taylor_Green_Vortex/time_iteration.f90:781).

The CUDA library is mandatory: ``load()`` raises if ``libsph_b200.so`` is not
built or no CUDA device is usable; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsph_b200.so")

# ---- constants mirrored from include/sph_b200.h ---------------------------
SPH_OK = 0
ERRORS = {
    -1: "SPH_E_ARG", -2: "SPH_E_CAPACITY", -3: "SPH_E_NONFINITE", -5: "SPH_E_CUDA",
    -6: "SPH_E_TIMEOUT", -7: "SPH_E_CONFIG", -8: "SPH_E_DOMAIN", -9: "SPH_E_SKIN",
    -10: "SPH_E_NODEVICE",
}
KERNEL_GAUSSIAN = 4
KERNEL_WENDLAND2 = 5
SOLVER_MODLR_DELTA_SPS = 0
SOLVER_MUSCL_DELTA_SPS = 1
SOLVER_MS_MODLR_DELTA = 2
SOLVER_MS_HLLC_DELTA = 3
SOLVER_DELTA_SPS = 4          # Solver_Normalized_Delta_SPH_SPS (the plain Taylor-Green method)
INTEGRATOR_RK4_REUSE = 0
INTEGRATOR_EULER_PC = 1
EOS_TAIT = 0
EOS_LINEAR = 1
PAIRS_ONE_FLUID = 0
PAIRS_NO_SAME_BND = 1
PREC_FP64 = 0
PREC_MIXED = 1
TYPE_WATER = 2
TYPE_PERIODIC = -101
TYPE_ILL = 120
TYPE_FIX_GHOST = -3
TYPE_BODY = -4
LOSS_VELOCITY_MISFIT = 0
LOSS_KINETIC_ENERGY = 1
LOSS_DRAG = 2
ADJ_NPARAMS = 1

EXPORTED_SYMBOLS = (
    "sph_init", "sph_free", "sph_set_state", "sph_get_state", "sph_find_particle_pair",
    "sph_rhs", "sph_step", "sph_diagnostics", "sph_get_timings", "sph_reset_timings",
    "sph_strerror", "sph_get_field", "sph_update_state", "sph_find_particle_pair_noalloc",
    "sph_set_initial_type", "sph_adjoint_forward", "sph_adjoint_backward",
    "sph_set_boundary_labels", "sph_set_body_motion", "sph_set_time", "sph_adjoint_motion_gradient",
    "sph_snapshot_begin", "sph_snapshot_query", "sph_snapshot_wait", "sph_restart_size", "sph_restart_save",
    "sph_restart_load",
)


class SphConfig(ctypes.Structure):
    _fields_ = [
        ("kernel_model", ctypes.c_int), ("solver", ctypes.c_int), ("eos", ctypes.c_int),
        ("pair_rule", ctypes.c_int), ("precision", ctypes.c_int), ("renormalize", ctypes.c_int),
        ("reference_literals", ctypes.c_int), ("periodic", ctypes.c_int), ("shifting", ctypes.c_int),
        ("integrator", ctypes.c_int),
        ("kernel_scale", ctypes.c_double), ("h", ctypes.c_double), ("dx", ctypes.c_double),
        ("rho0", ctypes.c_double), ("c0sq", ctypes.c_double), ("background_p", ctypes.c_double),
        ("nu", ctypes.c_double), ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
        ("fai", ctypes.c_double), ("delta", ctypes.c_double), ("delta_alpha", ctypes.c_double),
        ("xsph_eps", ctypes.c_double), ("shift_beta", ctypes.c_double), ("shift_R", ctypes.c_double),
        ("shift_max", ctypes.c_double), ("shift_n", ctypes.c_int), ("fs_threshold", ctypes.c_double),
        ("box_lo", ctypes.c_double * 2), ("box_hi", ctypes.c_double * 2),
        ("grid_lo", ctypes.c_double * 2), ("grid_hi", ctypes.c_double * 2),
        ("cell_skin", ctypes.c_double), ("laplacian", ctypes.c_int), ("free_surface", ctypes.c_int),
        ("mls_order", ctypes.c_int), ("mls_every", ctypes.c_int), ("mls_alpha", ctypes.c_double),
        ("ghost_assign", ctypes.c_int), ("wall_bc", ctypes.c_int), ("ghost_h_factor", ctypes.c_double),
        ("shock_release_time", ctypes.c_double), ("gravity", ctypes.c_double * 2),
    ]

    def copy(self) -> "SphConfig":
        c = SphConfig()
        ctypes.pointer(c)[0] = self
        return c


class SphDiag(ctypes.Structure):
    _fields_ = [
        ("kinetic_energy", ctypes.c_double), ("max_speed", ctypes.c_double),
        ("pair_count", ctypes.c_longlong), ("n_images", ctypes.c_int), ("n_surface", ctypes.c_int),
        ("body_force", ctypes.c_double * 6),
    ]


class SphAdjConfig(ctypes.Structure):
    _fields_ = [
        ("nsteps", ctypes.c_int), ("checkpoint_every", ctypes.c_int), ("loss", ctypes.c_int),
        ("reserved", ctypes.c_int), ("dt", ctypes.c_double), ("target_vel", ctypes.POINTER(ctypes.c_double)),
        ("body_motion", ctypes.POINTER(ctypes.c_double)),
    ]


class SphTimings(ctypes.Structure):
    _fields_ = [
        ("sort_ms", ctypes.c_double), ("pass_a_ms", ctypes.c_double), ("surface_ms", ctypes.c_double),
        ("pass_c_ms", ctypes.c_double), ("update_ms", ctypes.c_double), ("images_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double), ("rhs_evaluations", ctypes.c_longlong), ("steps", ctypes.c_longlong),
        ("kernel_launches", ctypes.c_longlong), ("adjoint_ms", ctypes.c_double),
    ]


# ---------------------------------------------------------------------------
# Configurations (values of information_module and of the benchmark cases)
# ---------------------------------------------------------------------------
def tgv_reference_config(n_side: int = 100) -> SphConfig:
    """The Taylor-Green case exactly as shipped in Taylor_Green_Vortex/information_module.f90:
    improved Gaussian (kernel_scale 3, :132-134), h = 1.2 dx, rho0 = 1000 (:30),
    c0^2 = 100 U (:142), nu = 1.0E-2 as a default real (:37), alpha 0, beta 2, fai 0.1,
    delta 0.1, Delta_alpha 0.02 (:245-256), shifting on (:346-350), renormalisation
    discarded, the default-real literals, periodic unit box."""
    dx = 1.0 / n_side
    c = SphConfig()
    c.kernel_model = KERNEL_GAUSSIAN
    c.solver = SOLVER_MODLR_DELTA_SPS
    c.eos = EOS_TAIT
    c.pair_rule = PAIRS_ONE_FLUID
    c.precision = PREC_FP64
    c.renormalize = 0
    c.reference_literals = 1
    c.periodic = 1
    c.shifting = 1
    c.integrator = 0
    c.kernel_scale = 3.0
    c.h = 1.20 * dx
    c.dx = dx
    c.rho0 = 1000.0
    c.c0sq = 100.0
    c.background_p = 0.0
    c.nu = float(np.float32(1.0e-2))
    c.alpha, c.beta, c.fai = 0.0, 2.0, 0.1
    c.delta, c.delta_alpha = 0.1, 0.02
    c.xsph_eps = 0.0
    c.shift_beta, c.shift_R, c.shift_max, c.shift_n = 0.5, 0.2, 0.25 * dx, 4
    c.fs_threshold = 0.65
    c.box_lo[:] = [0.0, 0.0]
    c.box_hi[:] = [1.0, 1.0]
    pad = 0.05
    c.grid_lo[:] = [-pad, -pad]
    c.grid_hi[:] = [1.0 + pad, 1.0 + pad]
    c.cell_skin = 0.1
    c.laplacian = 1
    c.free_surface = 1
    # Reinitialize_particle_density: quadratic MLS every 20 steps (:324-332),
    # slighted_modified_alpha = 0.0001 as a default real (:359)
    c.mls_order, c.mls_every, c.mls_alpha = 6, 20, float(np.float32(1.0e-4))
    return c


def tgv_baseline_config(n_side: int, solver: int = SOLVER_MUSCL_DELTA_SPS,
                        precision: int = PREC_FP64) -> SphConfig:
    """The Taylor-Green benchmark case: periodic unit square, Wendland C2 (support 2h,
    model 5 of Moving_Square.../Compute_Kernel.f90:172-198), h = 1.3 dx, rho0 = 1, U0 = 1,
    c0 = 10 U0, Re = 100 (nu = 0.01), Tait gamma 7, true 2x2 renormalisation,
    exact double constants."""
    dx = 1.0 / n_side
    c = tgv_reference_config(n_side)
    c.kernel_model = KERNEL_WENDLAND2
    c.solver = solver
    c.precision = precision
    c.renormalize = 1
    c.reference_literals = 0
    c.kernel_scale = 2.0
    c.h = 1.3 * dx
    c.rho0 = 1.0
    c.c0sq = 100.0
    c.nu = 0.01
    c.shift_max = 0.25 * dx
    c.cell_skin = 0.1
    c.mls_order = 0              # the benchmark case: no density re-initialisation
    return c


def baseline_dt(cfg: SphConfig) -> float:
    """Time step of the benchmark case: the acoustic CFL dt = 0.25 h / c0, limited by
    the viscous (Morris) criterion 0.125 h^2 / nu the reference combines it with
    (Taylor_Green_Vortex/Initialize_SPH_Calculation.f90:452-463, there with a fixed
    water viscosity).  At 2048^2 and Re = 100 the acoustic step alone gives
    nu dt / h^2 = 0.39, outside the explicit stability range of the Laplacian."""
    return min(0.25 * cfg.h / math.sqrt(cfg.c0sq), 0.125 * cfg.h * cfg.h / cfg.nu)


def tgv_lattice(n_side: int, U: float = 1.0, rho0: float = 1.0, c0sq: float = 100.0,
                sign: int = -1, reference_literals: bool = False):
    """Taylor-Green lattice of Taylor_Green_Vortex/Distribute_Initial_Particle.f90:206-231,
    vectorised.  sign=+1 is the reference's field (u = U sin cos, p = +rho0 U^2/4 ...),
    sign=-1 the benchmark's (u = -U cos sin, p = -rho0 U^2/4 ...).  Returns
    (pos[2n], vel[2n], rho[n], mass[n], press[n]) in Fortran column-major order."""
    PI = 3.14159265358979324
    dx = 1.0 / n_side
    j = np.arange(1, n_side + 1, dtype=np.float64)
    i = np.arange(1, n_side + 1, dtype=np.float64)
    X = (j - 1) * dx + dx / 2.0
    Y = (i - 1) * dx + dx / 2.0
    x = np.tile(X, n_side)
    y = np.repeat(Y, n_side)
    if sign > 0:
        u = U * np.sin(2 * PI * x) * np.cos(2 * PI * y)
        v = -U * np.cos(2 * PI * x) * np.sin(2 * PI * y)
        p = 0.25 * rho0 * (U * U) * (np.cos(4 * PI * x) + np.cos(4 * PI * y))
    else:
        u = -U * np.cos(2 * PI * x) * np.sin(2 * PI * y)
        v = U * np.sin(2 * PI * x) * np.cos(2 * PI * y)
        p = -0.25 * rho0 * (U * U) * (np.cos(4 * PI * x) + np.cos(4 * PI * y))
    ex = float(np.float32(0.142857142)) if reference_literals else 1.0 / 7.0
    rho = rho0 * np.power(1 + 7 * p / (c0sq * rho0), ex)
    mass = dx * dx * rho
    pos = np.concatenate([x, y])
    vel = np.concatenate([u, v])
    return pos, vel, rho, mass, p


# ---------------------------------------------------------------------------
# Library loading
# ---------------------------------------------------------------------------
_lib = None


class SphError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        msg = ERRORS.get(code, str(code))
        try:
            if _lib is not None:
                msg = _lib.sph_strerror(code).decode()
        except Exception:
            pass
        super().__init__(f"{where}: {msg} ({code})")


def _dp():
    return ctypes.POINTER(ctypes.c_double)


def load(path: str = LIB_PATH):
    """Load libsph_b200.so (raises if it is missing: the CUDA path is the only path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libsph_b200.so not built ({path}); run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    dp = _dp()
    ip = ctypes.POINTER(ctypes.c_int)
    lib.sph_init.argtypes = [ctypes.POINTER(SphConfig), ctypes.c_int, ctypes.POINTER(P)]
    lib.sph_free.argtypes = [P]
    lib.sph_set_state.argtypes = [P, ctypes.c_int, dp, dp, dp, dp, ip, dp]
    lib.sph_get_state.argtypes = [P, ctypes.c_int, dp, dp, dp, dp]
    lib.sph_update_state.argtypes = [P, ctypes.c_int, dp, dp, dp]
    lib.sph_set_initial_type.argtypes = [P, ctypes.c_int, ip]
    lib.sph_find_particle_pair.argtypes = [P, ctypes.c_longlong, ip, ip, dp, dp, ctypes.POINTER(ctypes.c_longlong)]
    lib.sph_rhs.argtypes = [P, dp, dp, dp, ip, ip]
    lib.sph_step.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.POINTER(SphDiag)]
    lib.sph_diagnostics.argtypes = [P, ctypes.POINTER(SphDiag)]
    lib.sph_get_timings.argtypes = [P, ctypes.POINTER(SphTimings)]
    lib.sph_reset_timings.argtypes = [P]
    lib.sph_get_field.argtypes = [P, ctypes.c_int, dp]
    lib.sph_set_boundary_labels.argtypes = [P, ctypes.c_int, ip]
    lib.sph_set_body_motion.argtypes = [P, dp, dp]
    lib.sph_set_time.argtypes = [P, ctypes.c_double]
    lib.sph_adjoint_forward.argtypes = [P, ctypes.POINTER(SphAdjConfig), dp]
    lib.sph_adjoint_backward.argtypes = [P, ctypes.c_double, dp, dp, dp, dp]
    lib.sph_adjoint_motion_gradient.argtypes = [P, dp]
    lib.sph_snapshot_begin.argtypes = [P, ctypes.c_int, dp, dp, dp, dp]
    lib.sph_snapshot_query.argtypes = [P]
    lib.sph_snapshot_wait.argtypes = [P]
    lib.sph_restart_size.argtypes = [ctypes.c_int]
    lib.sph_restart_save.argtypes = [P, ctypes.c_void_p, ctypes.c_size_t]
    lib.sph_restart_load.argtypes = [P, ctypes.c_void_p, ctypes.c_size_t]
    lib.sph_find_particle_pair_noalloc.argtypes = [ctypes.POINTER(SphConfig), ctypes.c_int, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.POINTER(ctypes.c_longlong), ctypes.c_void_p]
    lib.sph_strerror.argtypes = [ctypes.c_int]
    lib.sph_strerror.restype = ctypes.c_char_p
    for name in EXPORTED_SYMBOLS:
        if name != "sph_strerror":
            getattr(lib, name).restype = ctypes.c_int
    lib.sph_restart_size.restype = ctypes.c_size_t
    _lib = lib
    return lib


def _ptr(a, ctype=ctypes.c_double):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def _check(code: int, where: str):
    if code != SPH_OK:
        raise SphError(code, where)


# field ids of sph_get_field
FIELD_FRA_V, FIELD_BINV, FIELD_TAU, FIELD_GRADS = 0, 1, 2, 3
_FIELD_WIDTH = {FIELD_FRA_V: 1, FIELD_BINV: 4, FIELD_TAU: 3, FIELD_GRADS: 8}


class Simulation:
    """One libsph_b200 handle: the device-resident state of the Fortran
    subdomain arrays plus the configuration."""

    def __init__(self, cfg: SphConfig, capacity: int):
        self.lib = load()
        self.cfg = cfg.copy()
        self.capacity = int(capacity)
        h = ctypes.c_void_p()
        _check(self.lib.sph_init(ctypes.byref(self.cfg), self.capacity, ctypes.byref(h)), "sph_init")
        self.h = h
        self.n = 0
        self._adj_steps = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.sph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- state --------------------------------------------------------------
    def set_state(self, pos, vel, rho, mass, type_, sps_mass=None):
        n = rho.shape[0]
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        type_ = np.ascontiguousarray(type_, dtype=np.int32)
        sm = None if sps_mass is None else np.ascontiguousarray(sps_mass, dtype=np.float64)
        _check(self.lib.sph_set_state(self.h, n, _ptr(pos), _ptr(vel), _ptr(rho), _ptr(mass),
                                      _ptr(type_, ctypes.c_int), _ptr(sm)), "sph_set_state")
        self.n = n

    def update_state(self, pos, vel, rho):
        """Host-side edit of x, v, rho between steps; keeps the K1 rates."""
        n = self.n
        _check(self.lib.sph_update_state(self.h, n, _ptr(np.ascontiguousarray(pos, np.float64)),
                                         _ptr(np.ascontiguousarray(vel, np.float64)),
                                         _ptr(np.ascontiguousarray(rho, np.float64))), "sph_update_state")

    def set_initial_type(self, itype):
        """subdomain_particle_initial_type (SPH_TYPE_BODY marks the body for the body force)."""
        it = np.ascontiguousarray(itype, dtype=np.int32)
        _check(self.lib.sph_set_initial_type(self.h, self.n, _ptr(it, ctypes.c_int)), "sph_set_initial_type")

    def set_boundary_labels(self, labels):
        """subdomain_Boundary_particle_type (-6 horizontal wall, -7 corner, -8 vertical wall, 0 other)."""
        lb = np.ascontiguousarray(labels, dtype=np.int32)
        _check(self.lib.sph_set_boundary_labels(self.h, self.n, _ptr(lb, ctypes.c_int)), "sph_set_boundary_labels")

    def set_body_motion(self, vel, acc=(0.0, 0.0)):
        """Custom_velocity / Custom_accleration of the body for the following steps."""
        v = np.ascontiguousarray(vel, np.float64)
        a = np.ascontiguousarray(acc, np.float64)
        _check(self.lib.sph_set_body_motion(self.h, _ptr(v), _ptr(a)), "sph_set_body_motion")

    def set_time(self, t: float):
        _check(self.lib.sph_set_time(self.h, float(t)), "sph_set_time")

    def snapshot_begin(self, pos, vel, rho, press):
        """Queue a copy of the state into the given float64 arrays (2n, 2n, n, n;
        any may be None) and return at once (sph_snapshot_begin).  The arrays
        must stay alive until snapshot_wait; page-locked arrays let the transfer
        overlap the following steps."""
        arrs = [pos, vel, rho, press]
        for a, m in zip(arrs, (2, 2, 1, 1)):
            if a is not None and (a.dtype != np.float64 or a.size != m * self.n or not a.flags.c_contiguous):
                raise ValueError("snapshot buffers: contiguous float64 arrays of 2n, 2n, n, n values")
        self._snap_keep = arrs
        _check(self.lib.sph_snapshot_begin(self.h, self.n, *[_ptr(a) if a is not None else None for a in arrs]),
               "sph_snapshot_begin")

    def snapshot_query(self) -> bool:
        """True when the last snapshot has arrived in its host buffers."""
        rc = self.lib.sph_snapshot_query(self.h)
        if rc < 0:
            _check(rc, "sph_snapshot_query")
        return rc == 0

    def snapshot_wait(self):
        _check(self.lib.sph_snapshot_wait(self.h), "sph_snapshot_wait")
        self._snap_keep = None

    def restart_save(self) -> bytes:
        """The exact restart image of the handle (sph_restart_save)."""
        size = self.lib.sph_restart_size(self.n)
        buf = ctypes.create_string_buffer(size)
        _check(self.lib.sph_restart_save(self.h, buf, size), "sph_restart_save")
        return buf.raw

    def restart_load(self, image: bytes):
        """Restore a restart image (sph_restart_load); n comes from the image."""
        buf = ctypes.create_string_buffer(image, len(image))
        _check(self.lib.sph_restart_load(self.h, buf, len(image)), "sph_restart_load")
        self.n = int(np.frombuffer(image[12:16], np.int32)[0])

    def get_state(self):
        n = self.n
        pos = np.empty(2 * n); vel = np.empty(2 * n); rho = np.empty(n); press = np.empty(n)
        _check(self.lib.sph_get_state(self.h, n, _ptr(pos), _ptr(vel), _ptr(rho), _ptr(press)), "sph_get_state")
        return pos, vel, rho, press

    # --- reference-named entry points ----------------------------------------
    def find_particle_pair(self, pair_cap: int, want_kernel: bool = True):
        pi = np.zeros(pair_cap, np.int32); pj = np.zeros(pair_cap, np.int32)
        w = np.zeros(pair_cap) if want_kernel else None
        dw = np.zeros(2 * pair_cap) if want_kernel else None
        cnt = ctypes.c_longlong(0)
        code = self.lib.sph_find_particle_pair(self.h, pair_cap, _ptr(pi, ctypes.c_int), _ptr(pj, ctypes.c_int),
                                               _ptr(w), _ptr(dw), ctypes.byref(cnt))
        _check(code, "sph_find_particle_pair")
        m = cnt.value
        out = {"pair_i": pi[:m], "pair_j": pj[:m], "pair_number": m}
        if want_kernel:
            out["w"] = w[:m]
            out["dwdx"] = np.stack([dw[:m], dw[pair_cap:pair_cap + m]])
        return out

    def single_step_compute(self):
        n = self.n
        drho = np.empty(n); acc = np.empty(2 * n); avg = np.empty(2 * n)
        fs = np.empty(n, np.int32); near = np.empty(n, np.int32)
        _check(self.lib.sph_rhs(self.h, _ptr(drho), _ptr(acc), _ptr(avg), _ptr(fs, ctypes.c_int),
                                _ptr(near, ctypes.c_int)), "sph_rhs")
        return {"drhodt": drho, "acc": acc, "avg_vel": avg, "fs": fs, "near": near}

    def field(self, fid: int):
        out = np.empty(_FIELD_WIDTH[fid] * self.n)
        _check(self.lib.sph_get_field(self.h, fid, _ptr(out)), "sph_get_field")
        return out

    def time_iteration(self, nsteps: int, dt: float) -> SphDiag:
        d = SphDiag()
        _check(self.lib.sph_step(self.h, int(nsteps), float(dt), ctypes.byref(d)), "sph_step")
        return d

    def diagnostics(self) -> SphDiag:
        d = SphDiag()
        _check(self.lib.sph_diagnostics(self.h, ctypes.byref(d)), "sph_diagnostics")
        return d

    def timings(self) -> SphTimings:
        t = SphTimings()
        _check(self.lib.sph_get_timings(self.h, ctypes.byref(t)), "sph_get_timings")
        return t

    def reset_timings(self):
        _check(self.lib.sph_reset_timings(self.h), "sph_reset_timings")

    def adjoint_forward(self, nsteps: int, dt: float, checkpoint_every: int = 32,
                        loss: int = LOSS_VELOCITY_MISFIT, target_vel=None, body_motion=None) -> float:
        """nsteps time steps with state checkpoints every checkpoint_every steps;
        returns the loss (sph_adjoint_forward).  body_motion: (nsteps, 4) per-step
        body velocity and acceleration, or None for the handle's constant motion."""
        a = SphAdjConfig()
        a.nsteps, a.checkpoint_every, a.loss, a.dt = int(nsteps), int(checkpoint_every), int(loss), float(dt)
        keep = motion = None
        if target_vel is not None:
            keep = np.ascontiguousarray(target_vel, np.float64)
            if keep.shape != (2 * self.n,):
                raise ValueError("target_vel must hold 2n values (u block, v block)")
            a.target_vel = keep.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        if body_motion is not None:
            motion = np.ascontiguousarray(body_motion, np.float64)
            if motion.shape != (int(nsteps), 4):
                raise ValueError("body_motion must have shape (nsteps, 4)")
            a.body_motion = motion.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        out = ctypes.c_double(0.0)
        _check(self.lib.sph_adjoint_forward(self.h, ctypes.byref(a), ctypes.byref(out)), "sph_adjoint_forward")
        self._adj_steps = int(nsteps)
        return out.value

    def adjoint_backward(self, dloss: float = 1.0) -> dict:
        """Gradient of dloss * loss with respect to the state the last
        adjoint_forward started from and to the viscosity."""
        n = self.n
        gv = np.zeros(2 * n); gx = np.zeros(2 * n); gr = np.zeros(n); gp = np.zeros(ADJ_NPARAMS)
        _check(self.lib.sph_adjoint_backward(self.h, float(dloss), _ptr(gv), _ptr(gr), _ptr(gx), _ptr(gp)),
               "sph_adjoint_backward")
        return {"vel0": gv, "rho0": gr, "pos0": gx, "nu": float(gp[0])}

    def adjoint_motion_gradient(self) -> np.ndarray:
        """dL/d(body_motion) of the last backward pass, shape (nsteps, 4)
        (sph_adjoint_motion_gradient)."""
        g = np.zeros(4 * self._adj_steps)
        _check(self.lib.sph_adjoint_motion_gradient(self.h, _ptr(g)), "sph_adjoint_motion_gradient")
        return g.reshape(self._adj_steps, 4)


@dataclass
class TgvCase:
    """A Taylor-Green initial state ready for Simulation.set_state."""
    cfg: SphConfig
    pos: np.ndarray
    vel: np.ndarray
    rho: np.ndarray
    mass: np.ndarray
    type: np.ndarray

    @property
    def n(self) -> int:
        return self.rho.shape[0]


def make_tgv(n_side: int, reference: bool = False, solver: int = SOLVER_MUSCL_DELTA_SPS,
             precision: int = PREC_FP64, jitter: float = 0.0, seed: int = 0) -> TgvCase:
    if reference:
        cfg = tgv_reference_config(n_side)
        pos, vel, rho, mass, _ = tgv_lattice(n_side, rho0=1000.0, c0sq=100.0, sign=+1, reference_literals=True)
    else:
        cfg = tgv_baseline_config(n_side, solver, precision)
        pos, vel, rho, mass, _ = tgv_lattice(n_side, rho0=1.0, c0sq=100.0, sign=-1)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        pos = pos + rng.uniform(-jitter, jitter, pos.shape) * cfg.dx
    typ = np.full(rho.shape[0], TYPE_WATER, np.int32)
    return TgvCase(cfg, pos, vel, rho, mass, typ)


def body_motion_schedule(coeffs, nsteps: int, dt: float, t0: float = 0.0, period: float = 1.0):
    """Per-step body motion for Simulation.adjoint_forward(body_motion=...) and its
    Jacobian with respect to the motion parameters.

    The body moves in x with u(t) = a_0 + sum_{k=1..K} a_k sin(2 pi k t / period)
    (a_0 alone is the impulsive start at constant speed; the reference's motion
    table is not part of its source tree), v = 0, evaluated at the times the steps
    use, t0 + (s + 1) dt.  Returns (schedule, jac): schedule[s] = (u, 0, du/dt, 0)
    with shape (nsteps, 4), and jac[s, :, k] = d schedule[s] / d a_k, so that
    dL/da = einsum('sq,sqk->k', adjoint_motion_gradient(), jac)."""
    a = np.asarray(coeffs, np.float64)
    t = t0 + (np.arange(int(nsteps)) + 1.0) * dt
    w = 2.0 * np.pi / period
    jac = np.zeros((int(nsteps), 4, a.size))
    jac[:, 0, 0] = 1.0
    for k in range(1, a.size):
        jac[:, 0, k] = np.sin(k * w * t)
        jac[:, 2, k] = k * w * np.cos(k * w * t)
    return jac @ a, jac


def fourier_perturbation(pos, n_modes: int = 8, amp: float = 0.05, seed: int = 0, kmax: int = 4,
                         box: float = 1.0) -> np.ndarray:
    """A divergence-free velocity perturbation on the periodic box: the curl of
    a sum of n_modes stream-function modes sin(2 pi (kx x + ky y)/L + phase)
    with random integer wave numbers 1..kmax, random phases and weights,
    scaled so that its largest speed is amp.  pos is the 2n column-major
    position array; returns 2n values (u block, v block)."""
    n = pos.shape[0] // 2
    x, y = pos[:n], pos[n:]
    rng = np.random.default_rng(seed)
    u = np.zeros(n); v = np.zeros(n)
    for _ in range(n_modes):
        kx, ky = rng.integers(1, kmax + 1, 2) * rng.choice([-1, 1], 2)
        ph = rng.uniform(0.0, 2.0 * np.pi)
        wgt = rng.uniform(0.5, 1.0)
        arg = 2.0 * np.pi * (kx * x + ky * y) / box + ph
        c = np.cos(arg) * wgt * 2.0 * np.pi / box
        u += c * ky          # d psi / dy
        v -= c * kx          # -d psi / dx
    scale = amp / max(np.sqrt(u * u + v * v).max(), 1e-300)
    return np.concatenate([u, v]) * scale


# ---------------------------------------------------------------------------
# Moving-square layout (SPHERIC test 6 geometry of Moving_Square.../Information_Module.f90,
# scaled): a water-filled tank with fixed ghost walls and a square body made of
# ghost particles whose initial type marks the body.
# ---------------------------------------------------------------------------
def moving_square_config(dx: float, lx: float, ly: float, solver: int = SOLVER_MS_HLLC_DELTA,
                         precision: int = PREC_FP64, re: float = 100.0, U: float = 1.0, D: float = 1.0,
                         c0: float = 10.0) -> SphConfig:
    """Improved Gaussian (model 4, kernel_scale 3) with h = 1.15 dx as the moving-square case
    ships (Information_Module.f90:615-616), linear (Tammann) EOS (:305), alpha 0.03, beta 2,
    epsilon 0.1 (:630-644), Morris laplacian (:303), no free surface (:285), Euler
    predictor-corrector (:699), max shift 0.15 dx (:679); rho0 = 1 and nu = U D / Re."""
    c = SphConfig()
    c.kernel_model = KERNEL_GAUSSIAN
    c.solver = solver
    c.eos = EOS_LINEAR
    c.pair_rule = PAIRS_NO_SAME_BND
    c.precision = precision
    c.renormalize = 0
    c.reference_literals = 1
    c.periodic = 0
    c.shifting = 1
    c.integrator = INTEGRATOR_EULER_PC
    c.kernel_scale = 3.0
    c.h = 1.15 * dx
    c.dx = dx
    c.rho0 = 1.0
    c.c0sq = c0 * c0
    c.background_p = 0.0
    c.nu = U * D / re
    c.alpha, c.beta, c.fai = 0.03, 2.0, 0.1
    c.delta, c.delta_alpha = 0.1, 0.02
    c.xsph_eps = 0.1
    c.shift_beta, c.shift_R, c.shift_max, c.shift_n = 0.5, 0.2, 0.15 * dx, 4
    c.fs_threshold = 0.65
    c.box_lo[:] = [0.0, 0.0]
    c.box_hi[:] = [lx, ly]
    pad = 6 * dx
    c.grid_lo[:] = [-pad, -pad]
    c.grid_hi[:] = [lx + pad, ly + pad]
    c.cell_skin = 0.1
    c.laplacian = 1
    c.free_surface = 0
    # Reinitialize_particle_density: linear MLS every 40 steps (:662-671),
    # Slighted_modified_alpha = 1e-5 (:782)
    c.mls_order, c.mls_every, c.mls_alpha = 3, 40, 1.0e-5
    # Assign_boundary_particles parameters: no slip (ExternalBoundaryCondition 0, :301),
    # average smoothing length 1.2 h, Shock_wave_release_time 10 (:715), no gravity.
    # ghost_assign = 0: the ghost states are the caller's (set ghost_assign = 1, the
    # labels and the body motion to let the library assign them every RHS).
    c.ghost_assign, c.wall_bc, c.ghost_h_factor, c.shock_release_time = 0, 0, 1.2, 10.0
    c.gravity[:] = [0.0, 0.0]
    return c


def moving_square_labels(case, itype) -> np.ndarray:
    """subdomain_Boundary_particle_type of a make_moving_square layout: wall ghosts
    below/above the tank within 0 <= x <= lx are horizontal (-6), left/right of it
    within 0 <= y <= ly vertical (-8), the corner blocks -7 (Initial_Particle_From_First_Step.f90:
    220-300); water and body particles 0 (the body's ghosts take its velocity)."""
    n = case.n
    x, y = case.pos[:n], case.pos[n:]
    lx, ly = case.cfg.box_hi[0], case.cfg.box_hi[1]
    lab = np.zeros(n, np.int32)
    wall = (case.type == TYPE_FIX_GHOST) & (np.asarray(itype) != TYPE_BODY)
    inx = (x >= 0.0) & (x <= lx)
    iny = (y >= 0.0) & (y <= ly)
    lab[wall & inx] = -6
    lab[wall & ~inx & iny] = -8
    lab[wall & ~inx & ~iny] = -7
    return lab


def make_moving_square(dx: float = 0.05, lx: float = 4.0, ly: float = 2.0, D: float = 0.5, U: float = 1.0,
                       layers: int = 4, solver: int = SOLVER_MS_HLLC_DELTA, precision: int = PREC_FP64,
                       jitter: float = 0.0, seed: int = 0):
    """Water lattice in [0,lx]x[0,ly] at rest (rho = rho0), `layers` rows of fixed ghost
    particles outside the walls, and a square body of side D centred at (lx/4, ly/2)
    whose ghost particles move with velocity (U, 0).  Returns (case, initial_type)."""
    cfg = moving_square_config(dx, lx, ly, solver, precision, U=U, D=D)
    xs = (np.arange(int(round(lx / dx))) + 0.5) * dx
    ys = (np.arange(int(round(ly / dx))) + 0.5) * dx
    X, Y = np.meshgrid(xs, ys)
    cx, cy = lx / 4, ly / 2
    inside = (np.abs(X - cx) < D / 2) & (np.abs(Y - cy) < D / 2)
    wx, wy = X[~inside], Y[~inside]
    gx = (np.arange(-layers, int(round(lx / dx)) + layers) + 0.5) * dx
    gy = (np.arange(-layers, int(round(ly / dx)) + layers) + 0.5) * dx
    GX, GY = np.meshgrid(gx, gy)
    wall = (GX < 0) | (GX > lx) | (GY < 0) | (GY > ly)
    bx, by = X[inside], Y[inside]
    x = np.concatenate([wx, GX[wall], bx])
    y = np.concatenate([wy, GY[wall], by])
    nw, ng, nb = wx.size, int(wall.sum()), bx.size
    typ = np.concatenate([np.full(nw, TYPE_WATER), np.full(ng + nb, TYPE_FIX_GHOST)]).astype(np.int32)
    ityp = np.concatenate([np.full(nw + ng, 0), np.full(nb, TYPE_BODY)]).astype(np.int32)
    ityp[:nw] = TYPE_WATER
    ityp[nw:nw + ng] = TYPE_FIX_GHOST
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        x[:nw] += rng.uniform(-jitter, jitter, nw) * dx
        y[:nw] += rng.uniform(-jitter, jitter, nw) * dx
    n = x.size
    u = np.zeros(n)
    v = np.zeros(n)
    u[nw + ng:] = U
    rho = np.full(n, cfg.rho0)
    mass = rho * dx * dx
    pos = np.concatenate([x, y])
    vel = np.concatenate([u, v])
    return TgvCase(cfg, pos, vel, rho, mass, typ), ityp
