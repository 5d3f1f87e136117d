"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the reference results to compare against.  The
product path never loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "sph-2d_b200"))
from sph_b200 import SphConfig  # noqa: E402  (struct layout only)

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    cp = ctypes.POINTER(SphConfig)
    lib.oracle_threads.argtypes = [ctypes.c_int]
    lib.oracle_threads.restype = ctypes.c_int
    lib.oracle_tgv_init.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp]
    lib.oracle_find_particle_pair.argtypes = [cp, ctypes.c_int, dp, ip, ctypes.c_longlong, ip, ip, dp, dp]
    lib.oracle_find_particle_pair.restype = ctypes.c_longlong
    lib.oracle_periodic_images.argtypes = [cp, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, ip, ip]
    lib.oracle_rhs.argtypes = [cp, ctypes.c_int, dp, dp, dp, dp, ip, dp, dp, dp, dp, ip, ip, dp, dp, dp, dp]
    lib.oracle_rhs.restype = ctypes.c_longlong
    lib.oracle_create.argtypes = [cp, ctypes.c_int, dp, dp, dp, dp, ip, dp]
    lib.oracle_create.restype = ctypes.c_void_p
    lib.oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
    lib.oracle_get_state.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, dp, dp, dp]
    lib.oracle_kinetic_energy.argtypes = [ctypes.c_void_p]
    lib.oracle_kinetic_energy.restype = ctypes.c_double
    lib.oracle_last_pair_count.argtypes = [ctypes.c_void_p]
    lib.oracle_last_pair_count.restype = ctypes.c_longlong
    lib.oracle_last_images.argtypes = [ctypes.c_void_p]
    lib.oracle_destroy.argtypes = [ctypes.c_void_p]
    lib.oracle_set_initial_type.argtypes = [ctypes.c_void_p, ctypes.c_int, ip]
    lib.oracle_body_force.argtypes = [ctypes.c_void_p, dp]
    lib.oracle_rhs_body_force.argtypes = [cp, ctypes.c_int, dp, dp, dp, dp, ip, ip, dp]
    lib.oracle_mls_reinit.argtypes = [cp, ctypes.c_int, dp, dp, dp, ip, dp]
    lib.oracle_set_ghost_state.argtypes = [ctypes.c_int, ip, dp, dp, ctypes.c_double]
    lib.oracle_tangent.argtypes = [cp, ctypes.c_int, dp, dp, dp, dp, ip, dp, dp, dp, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_int, dp, dp, dp, dp, dp]
    lib.oracle_tangent_ms.argtypes = [cp, ctypes.c_int, dp, dp, dp, dp, ip, ip, ip, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_double, dp, ctypes.c_int, dp, dp, dp, dp, ctypes.c_double, dp, dp]
    lib.oracle_set_muscl_gradient_scale.argtypes = [ctypes.c_double]
    lib.oracle_muscl_limiter.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, dp, dp]
    lib.oracle_hllc_state.argtypes = [cp, dp, dp]
    _lib = lib
    return lib


def _p(a, t=ctypes.c_double):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(t))


def threads(n: int = 0) -> int:
    return load().oracle_threads(n)


def tgv_init(nx, ny, U=1.0, rho0=1000.0, c0sq=100.0, sign=1, reference_literals=True):
    n = nx * ny
    pos = np.empty(2 * n); vel = np.empty(2 * n); rho = np.empty(n); mass = np.empty(n); press = np.empty(n)
    load().oracle_tgv_init(nx, ny, 1.0, 1.0, U, rho0, c0sq, sign, int(reference_literals),
                           _p(pos), _p(vel), _p(rho), _p(mass), _p(press))
    return pos, vel, rho, mass, press


def find_particle_pair(cfg: SphConfig, pos, type_, pair_cap=None):
    n = type_.shape[0]
    if pair_cap is None:
        pair_cap = 80 * n + 16
    pi = np.zeros(pair_cap, np.int32); pj = np.zeros(pair_cap, np.int32)
    w = np.zeros(pair_cap); dw = np.zeros(2 * pair_cap)
    pos = np.ascontiguousarray(pos, np.float64); type_ = np.ascontiguousarray(type_, np.int32)
    m = load().oracle_find_particle_pair(ctypes.byref(cfg), n, _p(pos), _p(type_, ctypes.c_int), pair_cap,
                                         _p(pi, ctypes.c_int), _p(pj, ctypes.c_int), _p(w), _p(dw))
    if m > pair_cap:
        raise RuntimeError("pair capacity exceeded")
    return {"pair_i": pi[:m], "pair_j": pj[:m], "w": w[:m],
            "dwdx": np.stack([dw[:m], dw[pair_cap:pair_cap + m]]), "pair_number": m}


def periodic_images(cfg: SphConfig, pos, vel, rho, mass, type_, cap=None):
    n = rho.shape[0]
    if cap is None:
        cap = 2 * n + 64
    P = np.zeros(2 * cap); V = np.zeros(2 * cap); R = np.zeros(cap); M = np.zeros(cap)
    T = np.zeros(cap, np.int32); S = np.full(cap, -1, np.int32)
    P[:n] = pos[:n]; P[cap:cap + n] = pos[n:]; V[:n] = vel[:n]; V[cap:cap + n] = vel[n:]
    R[:n] = rho; M[:n] = mass; T[:n] = type_
    m = load().oracle_periodic_images(ctypes.byref(cfg), n, cap, _p(P), _p(V), _p(R), _p(M),
                                      _p(T, ctypes.c_int), _p(S, ctypes.c_int))
    if m < 0:
        raise RuntimeError("image capacity exceeded")
    pos2 = np.concatenate([P[:m], P[cap:cap + m]]); vel2 = np.concatenate([V[:m], V[cap:cap + m]])
    return pos2, vel2, R[:m].copy(), M[:m].copy(), T[:m].copy(), S[:m].copy()


def rhs(cfg: SphConfig, pos, vel, rho, mass, type_, sps_mass=None):
    n = rho.shape[0]
    out = {k: np.zeros(n) for k in ("drhodt", "fra_v")}
    out["acc"] = np.zeros(2 * n); out["avg_vel"] = np.zeros(2 * n)
    out["fs"] = np.zeros(n, np.int32); out["near"] = np.zeros(n, np.int32)
    out["binv"] = np.zeros(4 * n); out["tau"] = np.zeros(3 * n); out["grads"] = np.zeros(8 * n)
    a = [np.ascontiguousarray(x, np.float64) for x in (pos, vel, rho, mass)]
    t = np.ascontiguousarray(type_, np.int32)
    sm = None if sps_mass is None else np.ascontiguousarray(sps_mass, np.float64)
    m = load().oracle_rhs(ctypes.byref(cfg), n, _p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]), _p(t, ctypes.c_int), _p(sm),
                          _p(out["drhodt"]), _p(out["acc"]), _p(out["avg_vel"]), _p(out["fs"], ctypes.c_int),
                          _p(out["near"], ctypes.c_int), _p(out["fra_v"]), _p(out["binv"]), _p(out["tau"]),
                          _p(out["grads"]))
    out["pair_number"] = m
    return out


class OracleSim:
    """The oracle's time_iteration on a copy of the given state."""

    def __init__(self, cfg: SphConfig, pos, vel, rho, mass, type_, sps_mass=None):
        self.lib = load()
        self.cfg = cfg.copy()
        self.n = rho.shape[0]
        a = [np.ascontiguousarray(x, np.float64) for x in (pos, vel, rho, mass)]
        t = np.ascontiguousarray(type_, np.int32)
        sm = None if sps_mass is None else np.ascontiguousarray(sps_mass, np.float64)
        self.h = self.lib.oracle_create(ctypes.byref(self.cfg), self.n, _p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]),
                                        _p(t, ctypes.c_int), _p(sm))

    def run(self, nsteps: int, dt: float):
        self.lib.oracle_run(self.h, int(nsteps), float(dt))

    def state(self):
        n = self.n
        pos = np.empty(2 * n); vel = np.empty(2 * n); rho = np.empty(n); press = np.empty(n)
        self.lib.oracle_get_state(self.h, n, _p(pos), _p(vel), _p(rho), _p(press))
        return pos, vel, rho, press

    def set_initial_type(self, itype):
        it = np.ascontiguousarray(itype, np.int32)
        self.lib.oracle_set_initial_type(self.h, self.n, _p(it, ctypes.c_int))

    def body_force(self):
        out = np.zeros(6)
        self.lib.oracle_body_force(self.h, _p(out))
        return out

    def kinetic_energy(self) -> float:
        return self.lib.oracle_kinetic_energy(self.h)

    def last_pair_count(self) -> int:
        return self.lib.oracle_last_pair_count(self.h)

    def last_images(self) -> int:
        return self.lib.oracle_last_images(self.h)

    def __del__(self):
        try:
            if self.h:
                self.lib.oracle_destroy(self.h)
                self.h = None
        except Exception:
            pass


def rhs_body_force(cfg: SphConfig, pos, vel, rho, mass, type_, itype):
    out = np.zeros(6)
    a = [np.ascontiguousarray(x, np.float64) for x in (pos, vel, rho, mass)]
    t = np.ascontiguousarray(type_, np.int32)
    it = np.ascontiguousarray(itype, np.int32)
    load().oracle_rhs_body_force(ctypes.byref(cfg), rho.shape[0], _p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]),
                                 _p(t, ctypes.c_int), _p(it, ctypes.c_int), _p(out))
    return out


def tangent(cfg: SphConfig, pos, vel, rho, mass, type_, nsteps: int, dt: float, dpos=None, dvel=None, drho=None,
            dnu: float = 0.0, loss: int = 0, target_vel=None):
    """FP64 tangent-linear model (sph_tangent.cpp): the loss of the state after
    nsteps steps, its derivative along (dpos, dvel, drho, dnu), and the final
    state.  loss 0: squared velocity misfit against target_vel, 1: kinetic energy."""
    n = rho.shape[0]
    a = [np.ascontiguousarray(x, np.float64) for x in (pos, vel, rho, mass)]
    t = np.ascontiguousarray(type_, np.int32)
    d = [None if x is None else np.ascontiguousarray(x, np.float64) for x in (dpos, dvel, drho)]
    tg = None if target_vel is None else np.ascontiguousarray(target_vel, np.float64)
    out = np.zeros(2)
    P = np.zeros(2 * n); V = np.zeros(2 * n); R = np.zeros(n)
    rc = load().oracle_tangent(ctypes.byref(cfg), n, _p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]), _p(t, ctypes.c_int),
                               _p(d[0]), _p(d[1]), _p(d[2]), float(dnu), int(nsteps), float(dt), int(loss), _p(tg),
                               _p(out), _p(P), _p(V), _p(R))
    if rc != 0:
        raise RuntimeError(f"oracle_tangent failed ({rc})")
    return out[0], out[1], (P, V, R)


def tangent_ms(cfg: SphConfig, pos, vel, rho, mass, type_, itype, labels, t0: float, nsteps: int, dt: float,
               motion, loss: int, target_vel=None, dpos=None, dvel=None, drho=None, dnu: float = 0.0, dmotion=None):
    """Moving-square FP64 tangent-linear model (sph_tangent.cpp, oracle_tangent_ms):
    the loss after nsteps Euler predictor-corrector steps with the per-step body
    motion (nsteps, 4) and its derivative along (dpos, dvel, drho, dnu, dmotion)."""
    n = rho.shape[0]
    a = [np.ascontiguousarray(x, np.float64) for x in (pos, vel, rho, mass)]
    ti = [np.ascontiguousarray(x, np.int32) for x in (type_, itype, labels)]
    mo = np.ascontiguousarray(motion, np.float64).reshape(-1)
    d = [None if x is None else np.ascontiguousarray(x, np.float64).reshape(-1) for x in (dpos, dvel, drho, dmotion)]
    tg = None if target_vel is None else np.ascontiguousarray(target_vel, np.float64)
    out = np.zeros(2)
    rc = load().oracle_tangent_ms(ctypes.byref(cfg), n, _p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]),
                                  _p(ti[0], ctypes.c_int), _p(ti[1], ctypes.c_int), _p(ti[2], ctypes.c_int),
                                  float(t0), int(nsteps), float(dt), _p(mo), int(loss), _p(tg), _p(d[0]), _p(d[1]),
                                  _p(d[2]), float(dnu), _p(d[3]), _p(out))
    if rc != 0:
        raise RuntimeError(f"oracle_tangent_ms failed ({rc})")
    return out[0], out[1]


def mls_reinit(cfg: SphConfig, pos, rho, mass, type_):
    """Reinitialize_particle_density applied once to the given particles."""
    n = rho.shape[0]
    out = np.zeros(n)
    a = [np.ascontiguousarray(x, np.float64) for x in (pos, rho, mass)]
    t = np.ascontiguousarray(type_, np.int32)
    rc = load().oracle_mls_reinit(ctypes.byref(cfg), n, _p(a[0]), _p(a[1]), _p(a[2]), _p(t, ctypes.c_int), _p(out))
    if rc != 0:
        raise RuntimeError("oracle_mls_reinit failed")
    return out


def set_ghost_state(labels, body_vel=(0.0, 0.0), body_acc=(0.0, 0.0), t: float = 0.0):
    """Wall labels, body velocity / acceleration and physical time for the
    oracle's ghost assignment (used when the configuration has ghost_assign = 1)."""
    lb = np.ascontiguousarray(labels, np.int32)
    bv = np.ascontiguousarray(body_vel, np.float64)
    ba = np.ascontiguousarray(body_acc, np.float64)
    load().oracle_set_ghost_state(lb.shape[0], _p(lb, ctypes.c_int), _p(bv), _p(ba), float(t))


def set_muscl_gradient_scale(scale: float):
    """Factor on the MUSCL reconstruction gradients (grad p, grad u, grad v) of
    the following oracle RHS evaluations; 1 is the solver as written."""
    load().oracle_set_muscl_gradient_scale(float(scale))


def muscl_limiter(di: float, dj: float, dij: float):
    li = ctypes.c_double(0.0); lj = ctypes.c_double(0.0)
    load().oracle_muscl_limiter(float(di), float(dj), float(dij), ctypes.byref(li), ctypes.byref(lj))
    return li.value, lj.value


def hllc_state(cfg: SphConfig, vi, vj, e, rho_i, rho_j, c_i, c_j, p_i, p_j):
    """The oracle's HLLC pair state (v*, P*) for one pair; e is the unit vector
    from particle i to particle j."""
    inp = np.array([vi[0], vi[1], vj[0], vj[1], e[0], e[1], rho_i, rho_j, c_i, c_j, p_i, p_j], np.float64)
    out = np.zeros(3)
    rc = load().oracle_hllc_state(ctypes.byref(cfg), _p(inp), _p(out))
    if rc != 0:
        raise RuntimeError("oracle_hllc_state failed")
    return out[:2].copy(), float(out[2])
