"""CPU oracle for the SPH giant-impact step — TEST INFRASTRUCTURE ONLY.

Loads ``oracle/liboracle.so`` (built from ``sph_oracle.cpp`` by ``oracle/Makefile``) through ctypes and
exposes numpy-friendly wrappers. Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package, as the checker and the timed CPU reference; the product never does.

The C++ restates the Integrity engine's reference arithmetic (sean-reid/BotheadStudios, ``integrity-engine``):
f32 functions follow ``shaders/sph_step.wgsl`` and ``shaders/bh_gravity.wgsl``; f64 functions follow
``crates/engine/src/{hydrostatic,eos,bhtree,neighbors,atmosphere}.rs`` and ``tools/sph-verify/src/main.rs``.
Each C++ function cites the file:line it follows. The reference has no golden-vector files; the oracle is
pinned against the reference's own known-answer tests in ``tests/test_oracle_pins.py``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")
_lib = None

f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (no-op when it is newer than the source)."""
    src = os.path.join(_HERE, "sph_oracle.cpp")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _SO


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_SO):
        build()
    L = C.CDLL(_SO)
    L.orc_pressure64.restype = C.c_double
    L.orc_pressure64.argtypes = [f64p, C.c_double, C.c_double]
    L.orc_sound_speed_sq64.restype = C.c_double
    L.orc_sound_speed_sq64.argtypes = [f64p, C.c_double, C.c_double]
    L.orc_sound_speed64_wgsl.restype = C.c_double
    L.orc_sound_speed64_wgsl.argtypes = [f64p, C.c_double, C.c_double, C.c_double]
    L.orc_pressure32.restype = C.c_float
    L.orc_pressure32.argtypes = [f32p, C.c_float, C.c_float, C.c_float]
    L.orc_sound_speed32.restype = C.c_float
    L.orc_sound_speed32.argtypes = [f32p, C.c_float, C.c_float, C.c_float, C.c_float]
    L.orc_eos32.argtypes = [f32p, u32p, f32p, f32p, C.c_int, C.c_float, C.c_float, f32p, f32p]
    L.orc_w64.restype = C.c_double
    L.orc_w64.argtypes = [C.c_int, C.c_double, C.c_double]
    L.orc_dw64.restype = C.c_double
    L.orc_dw64.argtypes = [C.c_int, C.c_double, C.c_double]
    L.orc_w32.restype = C.c_float
    L.orc_w32.argtypes = [C.c_int, C.c_float, C.c_float]
    L.orc_dw32.restype = C.c_float
    L.orc_dw32.argtypes = [C.c_int, C.c_float, C.c_float]
    L.orc_bbox32.argtypes = [f32p, C.c_int, f32p, f32p]
    L.orc_morton32.argtypes = [f32p, C.c_int, f32p, f32p, u32p]
    L.orc_sort_code_index.argtypes = [u32p, C.c_int, u32p, u32p]
    L.orc_karras.argtypes = [u32p, C.c_int, u32p, u32p, u32p, C.c_int]
    L.orc_verify_tree.restype = C.c_int
    L.orc_verify_tree.argtypes = [u32p, u32p, u32p, C.c_int]
    L.orc_moments32.argtypes = [f32p, C.c_int, C.c_int, C.c_int, u32p, u32p, f32p, f32p, f32p]
    L.orc_gravity_bh32.restype = C.c_int
    L.orc_gravity_bh32.argtypes = [f32p, C.c_int, C.c_int, C.c_int, u32p, u32p, f32p, f32p, f32p, u32p,
                                   C.c_float, C.c_float, C.c_float, f32p]
    L.orc_gravity_direct32.argtypes = [f32p, C.c_int, C.c_float, C.c_float, f32p]
    L.orc_gravity_direct64.argtypes = [f64p, f64p, C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_double, f64p,
                                       C.c_int]
    L.orc_bhtree64.restype = C.c_int
    L.orc_bhtree64.argtypes = [f64p, f64p, C.c_int, C.c_double, C.c_double, C.c_double, f64p, C.c_int]
    L.orc_neighbours32.restype = C.c_longlong
    L.orc_neighbours32.argtypes = [f32p, C.c_int, u32p, u32p, C.c_int]
    L.orc_density32.argtypes = [f32p, f32p, C.c_int, C.c_int, f32p]
    L.orc_sph_forces32.argtypes = [f32p, f32p, f32p, f32p, f32p, f32p, C.c_int, C.c_float, C.c_float, C.c_float,
                                   C.c_int, f32p]
    L.orc_cpu_forces64.argtypes = [f64p, f64p, f64p, f64p, f64p, i32p, C.c_int, f64p, C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_double, C.c_int, f64p, f64p, f64p]
    L.orc_cpu_kdk64.argtypes = [f64p, f64p, f64p, f64p, f64p, i32p, C.c_int, f64p, C.c_double, C.c_double,
                                C.c_double, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int]
    L.orc_hydro_new.restype = C.c_void_p
    L.orc_hydro_new.argtypes = [C.c_int, f64p, f64p, f64p, f64p, f64p, i32p, f64p, C.c_int, C.c_double,
                                C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]
    L.orc_hydro_free.argtypes = [C.c_void_p]
    L.orc_hydro_step.argtypes = [C.c_void_p, C.c_double, C.c_int]
    L.orc_hydro_density.argtypes = [C.c_void_p, C.c_int]
    L.orc_hydro_forces.argtypes = [C.c_void_p, f64p, f64p, C.c_int]
    L.orc_hydro_eval_sampled.argtypes = [C.c_void_p, C.c_int, f64p]
    L.orc_hydro_courant_dt.restype = C.c_double
    L.orc_hydro_courant_dt.argtypes = [C.c_void_p, C.c_double, C.c_double]
    L.orc_hydro_get.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_max_threads.restype = C.c_int
    L.orc_conservation64.argtypes = [f64p, f64p, f64p, f64p, C.c_int, C.c_double, C.c_double, C.c_int, f64p]
    L.orc_h_solve32.restype = C.c_float
    L.orc_h_solve32.argtypes = [f32p, f32p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, f32p, f32p, f32p]
    L.orc_h_solve64.restype = C.c_int
    L.orc_h_solve64.argtypes = [f64p, f64p, f64p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                f64p, f64p, f64p]
    L.orc_relax32.argtypes = [f32p, f32p, f32p, C.c_int, C.c_float, C.c_float, C.c_float]
    L.orc_signal32.argtypes = [f32p, f32p, f32p, C.c_int, C.c_float, f32p]
    _lib = L
    return L


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ---- EOS ---------------------------------------------------------------------------------------------
def pressure64(eos10, rho, u):
    return lib().orc_pressure64(_c(eos10, np.float64), float(rho), float(u))


def sound_speed_sq64(eos10, rho, u):
    return lib().orc_sound_speed_sq64(_c(eos10, np.float64), float(rho), float(u))


def sound_speed64_wgsl(eos10, rho, u, du_floor=1.0):
    return lib().orc_sound_speed64_wgsl(_c(eos10, np.float64), float(rho), float(u), float(du_floor))


def pressure32(eos12, rho, u, rho_floor=1e-9):
    return lib().orc_pressure32(_c(eos12, np.float32), rho, u, rho_floor)


def sound_speed32(eos12, rho, u, du_floor=1.0, rho_floor=1e-9):
    return lib().orc_sound_speed32(_c(eos12, np.float32), rho, u, du_floor, rho_floor)


def eos32(eos_table12, mat, rho, u, du_floor=1.0, rho_floor=1e-9):
    n = len(rho)
    P = np.empty(n, np.float32)
    c = np.empty(n, np.float32)
    lib().orc_eos32(_c(eos_table12, np.float32).reshape(-1), _c(mat, np.uint32), _c(rho, np.float32),
                    _c(u, np.float32), n, du_floor, rho_floor, P, c)
    return P, c


# ---- tree --------------------------------------------------------------------------------------------
def bbox32(pos4):
    p = _c(pos4, np.float32)
    lo = np.empty(3, np.float32)
    hi = np.empty(3, np.float32)
    lib().orc_bbox32(p, len(p), lo, hi)
    return lo, hi


def morton32(pos4, lo, hi):
    p = _c(pos4, np.float32)
    codes = np.empty(len(p), np.uint32)
    lib().orc_morton32(p, len(p), _c(lo, np.float32), _c(hi, np.float32), codes)
    return codes


def sort_code_index(codes):
    codes = _c(codes, np.uint32)
    order = np.empty(len(codes), np.uint32)
    sc = np.empty(len(codes), np.uint32)
    lib().orc_sort_code_index(codes, len(codes), order, sc)
    return order, sc


def karras(leaf_codes, exact_dups=False):
    lc = _c(leaf_codes, np.uint32)
    L = len(lc)
    nn = 2 * L - 1
    left = np.zeros(max(L - 1, 1), np.uint32)
    right = np.zeros(max(L - 1, 1), np.uint32)
    parent = np.zeros(nn, np.uint32)
    lib().orc_karras(lc, L, left, right, parent, int(exact_dups))
    return left[: L - 1], right[: L - 1], parent


def verify_tree(left, right, parent, L):
    return bool(lib().orc_verify_tree(_c(left, np.uint32) if len(left) else np.zeros(1, np.uint32),
                                      _c(right, np.uint32) if len(right) else np.zeros(1, np.uint32),
                                      _c(parent, np.uint32), L))


def moments32(sbodies4, K, left, right):
    sb = _c(sbodies4, np.float32)
    n = len(sb)
    L = (n + K - 1) // K
    nn = 2 * L - 1
    com = np.zeros((nn, 4), np.float32)
    bmin = np.zeros((nn, 4), np.float32)
    bmax = np.zeros((nn, 4), np.float32)
    lft = _c(left, np.uint32) if len(left) else np.zeros(1, np.uint32)
    rgt = _c(right, np.uint32) if len(right) else np.zeros(1, np.uint32)
    lib().orc_moments32(sb, n, K, L, lft, rgt, com, bmin, bmax)
    return com, bmin, bmax


def gravity_bh32(sbodies4, K, left, right, com, bmin, bmax, order, theta, soft2, G):
    sb = _c(sbodies4, np.float32)
    n = len(sb)
    L = (n + K - 1) // K
    acc = np.zeros((n, 4), np.float32)
    lft = _c(left, np.uint32) if len(left) else np.zeros(1, np.uint32)
    rgt = _c(right, np.uint32) if len(right) else np.zeros(1, np.uint32)
    dropped = lib().orc_gravity_bh32(sb, n, K, L, lft, rgt, _c(com, np.float32), _c(bmin, np.float32),
                                     _c(bmax, np.float32), _c(order, np.uint32), theta, soft2, G, acc)
    return acc, dropped


def tree_pipeline32(bodies4, K=1, theta=0.5, soft=0.0, G=6.674e-11, exact_dups=False):
    """bbox → Morton → (code,index) sort → cluster codes → Karras → moments → traversal, all in f32.

    Mirrors the staged pipeline of tools/gpu-bh-verify (build_tree + cs_gravity_bh). Returns a dict with
    every intermediate so each stage can be compared separately.
    """
    b = _c(bodies4, np.float32)
    n = len(b)
    lo, hi = bbox32(b)
    codes = morton32(b, lo, hi)
    order, scodes = sort_code_index(codes)
    L = (n + K - 1) // K
    leaf_codes = scodes[np.arange(L) * K]
    left, right, parent = karras(leaf_codes, exact_dups)
    sb = np.ascontiguousarray(b[order])
    com, bmin, bmax = moments32(sb, K, left, right)
    acc, dropped = gravity_bh32(sb, K, left, right, com, bmin, bmax, order, theta,
                                np.float32(soft) * np.float32(soft), G)
    return dict(lo=lo, hi=hi, codes=codes, order=order, sorted_codes=scodes, leaf_codes=leaf_codes, left=left,
                right=right, parent=parent, sbodies=sb, com=com, bmin=bmin, bmax=bmax, acc=acc, dropped=dropped,
                L=L)


def gravity_direct32(bodies4, soft2, G):
    b = _c(bodies4, np.float32)
    acc = np.zeros((len(b), 4), np.float32)
    lib().orc_gravity_direct32(b, len(b), soft2, G, acc)
    return acc


def gravity_direct64(pos3, mass, soft, G, targets=None, nthreads=0):
    p = _c(pos3, np.float64)
    m = _c(mass, np.float64)
    n = len(m)
    if targets is None:
        nt, tp = n, None
    else:
        t = _c(targets, np.int32)
        nt, tp = len(t), t.ctypes.data_as(C.c_void_p)
    acc = np.zeros((nt, 3), np.float64)
    nthreads = nthreads or lib().orc_max_threads()
    lib().orc_gravity_direct64(p, m, n, tp, nt, soft, G, acc, nthreads)
    return acc


def bhtree64(pos3, mass, theta, soft, G, nthreads=1):
    p = _c(pos3, np.float64)
    acc = np.zeros((len(p), 3), np.float64)
    nodes = lib().orc_bhtree64(p, _c(mass, np.float64), len(p), theta, soft, G, acc, nthreads)
    return acc, nodes


# ---- SPH ---------------------------------------------------------------------------------------------
def neighbours32(pos4, cap=512):
    p = _c(pos4, np.float32)
    n = len(p)
    counts = np.zeros(n, np.uint32)
    lists = np.zeros(n * cap, np.uint32)
    tot = lib().orc_neighbours32(p, n, counts, lists, cap)
    if tot < 0:
        raise ValueError("neighbour cap exceeded")
    lists = lists.reshape(n, cap)
    return [lists[i, : counts[i]].copy() for i in range(n)]


def density32(pos4, mass, kernel=0):
    p = _c(pos4, np.float32)
    rho = np.empty(len(p), np.float32)
    lib().orc_density32(p, _c(mass, np.float32), len(p), kernel, rho)
    return rho


def sph_forces32(pos4, vel4, mass, rho, P, c, av_alpha=1.0, av_beta=2.0, r_min=1e-9, kernel=0):
    p = _c(pos4, np.float32)
    out = np.empty((len(p), 4), np.float32)
    lib().orc_sph_forces32(p, _c(vel4, np.float32), _c(mass, np.float32), _c(rho, np.float32), _c(P, np.float32),
                           _c(c, np.float32), len(p), av_alpha, av_beta, r_min, kernel, out)
    return out


def h_solve32(pos4, mass, eta, skin, iters, kernel=1):
    """The smoothing-length solve in f32: `iters` Jacobi-Newton steps from h0 = pos4[:, 3] inside the list skin,
    then the density at the final h. Returns (h, rho, residual) per particle."""
    p = _c(pos4, np.float32)
    n = len(p)
    h = np.empty(n, np.float32)
    rho = np.empty(n, np.float32)
    res = np.empty(n, np.float32)
    lib().orc_h_solve32(p, _c(mass, np.float32), n, kernel, eta, skin, int(iters), h, rho, res)
    return h, rho, res


def h_solve64(pos3, h0, mass, eta, skin, kernel=1, step_tol=1e-12, max_iter=200):
    """The same solve in f64, iterated until no h moves by more than step_tol in a step (Price 2012 Newton on
    rho(h) = m (eta/h)^3 with the symmetric h_ij). Returns (h, rho, residual, steps); steps > max_iter means it
    did not settle."""
    n = len(mass)
    h = np.empty(n)
    rho = np.empty(n)
    res = np.empty(n)
    it = lib().orc_h_solve64(_c(pos3, np.float64), _c(h0, np.float64), _c(mass, np.float64), n, kernel, eta, skin,
                             step_tol, int(max_iter), h, rho, res)
    return h, rho, res, it


def relax32(pos4, vel4, acc4, dt, damp, omega):
    """One cs_relax step (sph_step.wgsl:245-257) in f32 on copies of pos4/vel4; returns (pos4, vel4)."""
    p = np.array(pos4, np.float32, order="C")
    v = np.array(vel4, np.float32, order="C")
    lib().orc_relax32(p, v, _c(acc4, np.float32), len(p), dt, damp, omega)
    return p, v


def signal32(pos4, vel4, c, floor=1.0):
    """cs_signal (sph_step.wgsl:263-269): h / max(c + |v|, floor) per particle; the adaptive dt is cfl * min."""
    p = _c(pos4, np.float32)
    sig = np.empty(len(p), np.float32)
    lib().orc_signal32(p, _c(vel4, np.float32), _c(c, np.float32), len(p), floor, sig)
    return sig


def cpu_forces64(pos3, vel3, h, mass, u, mat, eos10_table, soft, G=6.674e-11, av_alpha=1.0, av_beta=2.0,
                 du_floor=1.0, kernel=0):
    n = len(h)
    rho = np.empty(n)
    acc = np.empty((n, 3))
    dudt = np.empty(n)
    lib().orc_cpu_forces64(_c(pos3, np.float64), _c(vel3, np.float64), _c(h, np.float64), _c(mass, np.float64),
                           _c(u, np.float64), _c(mat, np.int32), n, _c(eos10_table, np.float64).reshape(-1), soft, G,
                           av_alpha, av_beta, du_floor, kernel, rho, acc, dudt)
    return rho, acc, dudt


def cpu_kdk64(pos3, vel3, h, mass, u, mat, eos10_table, soft, dt, steps, G=6.674e-11, av_alpha=1.0, av_beta=2.0,
              du_floor=1.0, kernel=0):
    pos = np.array(pos3, np.float64, order="C")
    vel = np.array(vel3, np.float64, order="C")
    uu = np.array(u, np.float64)
    lib().orc_cpu_kdk64(pos, vel, _c(h, np.float64), _c(mass, np.float64), uu, _c(mat, np.int32), len(uu),
                        _c(eos10_table, np.float64).reshape(-1), soft, G, av_alpha, av_beta, du_floor, kernel, dt,
                        steps)
    return pos, vel, uu


class HydroBody:
    """Handle on the C++ restatement of ``HydroBody`` (hydrostatic.rs:241-374), f64."""

    def __init__(self, pos3, vel3, mass, u, h, mat, eos10_table, softening, G=6.674e-11, theta=0.5,
                 av_alpha=1.0, av_beta=2.0, kernel=0):
        self.n = len(mass)
        self._L = lib()
        eos = _c(eos10_table, np.float64).reshape(-1)
        self._h = self._L.orc_hydro_new(self.n, _c(pos3, np.float64), _c(vel3, np.float64), _c(mass, np.float64),
                                        _c(u, np.float64), _c(h, np.float64), _c(mat, np.int32), eos,
                                        len(eos) // 10, softening, G, theta, av_alpha, av_beta, kernel)

    def step(self, dt, nthreads=1):
        self._L.orc_hydro_step(self._h, dt, nthreads)

    def compute_density(self, nthreads=1):
        self._L.orc_hydro_density(self._h, nthreads)

    def forces_and_dudt(self, nthreads=1):
        acc = np.empty((self.n, 3))
        du = np.empty(self.n)
        self._L.orc_hydro_forces(self._h, acc, du, nthreads)
        return acc, du

    def eval_sampled(self, stride):
        """One force evaluation of the single-threaded path at full size with its per-particle loops run for
        every stride-th block of 512 consecutive particles: returns (seconds of the full-size parts, seconds of
        the sampled loops); a full evaluation takes about the first + stride x the second."""
        t = np.zeros(2)
        self._L.orc_hydro_eval_sampled(self._h, int(stride), t)
        return float(t[0]), float(t[1])

    def courant_dt(self, cfl, sig_floor=1.0):
        return self._L.orc_hydro_courant_dt(self._h, cfl, sig_floor)

    def state(self):
        pos = np.empty((self.n, 3))
        vel = np.empty((self.n, 3))
        u = np.empty(self.n)
        rho = np.empty(self.n)
        self._L.orc_hydro_get(self._h, pos.ctypes.data, vel.ctypes.data, u.ctypes.data, rho.ctypes.data)
        return pos, vel, u, rho

    def __del__(self):
        try:
            self._L.orc_hydro_free(self._h)
        except Exception:
            pass


def max_threads():
    return lib().orc_max_threads()


def conservation64(pos3, vel3, mass, u, soft=0.0, G=6.674e-11, with_pe=True):
    out = np.empty(9)
    lib().orc_conservation64(_c(pos3, np.float64), _c(vel3, np.float64), _c(mass, np.float64), _c(u, np.float64),
                             len(mass), soft, G, int(with_pe), out)
    return out


# ---- granular contact (particle_step.wgsl) ----------------------------------------------------------------
def dem_params(stiffness, normal_damp, friction, tangent_damp, cohesion, dt, gravity=(0.0, -9.81, 0.0)):
    return np.array([stiffness, normal_damp, friction, tangent_damp, cohesion, dt, *gravity], np.float32)


def dem_contacts32(pos3, vel3, radius, prm):
    L = lib()
    L.orc_dem_contacts32.argtypes = [f32p, f32p, f32p, C.c_int, f32p, f32p]
    n = len(radius)
    acc = np.zeros((n, 16), np.float32)
    L.orc_dem_contacts32(_c(pos3, np.float32), _c(vel3, np.float32), _c(radius, np.float32), n,
                         _c(prm, np.float32), acc)
    return acc


def dem_step32(pos3, vel3, radius, prm, substeps=1):
    """contacts + integrate, `substeps` times (the reference's dispatch without terrain/drag/cooling)."""
    L = lib()
    L.orc_dem_integrate32.argtypes = [f32p, f32p, f32p, C.c_int, f32p]
    pos = np.array(pos3, np.float32, order="C")
    vel = np.array(vel3, np.float32, order="C")
    for _ in range(substeps):
        acc = dem_contacts32(pos, vel, radius, prm)
        L.orc_dem_integrate32(pos, vel, acc, len(radius), _c(prm, np.float32))
    return pos, vel


# ---- learned smoothing-length MLP (FP64, optional BF16 operand rounding as in the product kernels) --------
def mlp_param_count(trainable: bool = False) -> int:
    L = lib()
    L.orc_mlp_param_count.restype = C.c_int
    return int(L.orc_mlp_param_count(1 if trainable else 0))


def mlp_forward(params, x, bf16: bool = True) -> np.ndarray:
    """De-normalised outputs (Δlog h) of the MLP for feature rows x[n][8]."""
    L = lib()
    L.orc_mlp_forward.argtypes = [f32p, f32p, C.c_int, C.c_int, f64p]
    x = _c(x, np.float32).reshape(-1, 8)
    out = np.zeros(len(x), np.float64)
    L.orc_mlp_forward(_c(params, np.float32), x, len(x), 1 if bf16 else 0, out)
    return out


def mlp_grad(params, x, t, bf16: bool = True):
    """(mean squared error on the normalised targets, its gradient w.r.t. the trainable parameters)."""
    L = lib()
    L.orc_mlp_grad.argtypes = [f32p, f32p, f32p, C.c_int, C.c_int, f64p]
    L.orc_mlp_grad.restype = C.c_double
    x = _c(x, np.float32).reshape(-1, 8)
    g = np.zeros(mlp_param_count(True), np.float64)
    loss = L.orc_mlp_grad(_c(params, np.float32), x, _c(t, np.float32), len(x), 1 if bf16 else 0, g)
    return float(loss), g


# ---- disk measurement and the Moon candidate (tools/impact-run/src/main.rs:732-878) -------------------
MEASURE_KEYS = ("earth_frac", "disk_mass", "disk_target", "disk_impactor", "remnant_target", "remnant_impactor",
                "escaped_target", "escaped_impactor", "r_remnant", "m_remnant", "clump_mass", "clump_target_frac",
                "clump_n", "n_clumps", "n_bound", "n_disk")


def measure_disk(particles, G, variant=0, remnant_frac=0.85, link_factor=2.0, roche=2.44, rho_fallback=2700.0,
                 pe_floor=1.0, pe_soft=1.0e4) -> dict:
    """The reference's disk measurement of one impact's 48-byte particle array (a dict keyed by MEASURE_KEYS):
    variant 0 = the impact-run tool's `measure`, variant 1 = the engine's `disk_stats_json`."""
    L = lib()
    L.orc_measure_disk.argtypes = [f32p, C.c_int, C.c_int] + [C.c_double] * 7 + [f64p]
    p = np.ascontiguousarray(np.ascontiguousarray(particles).view(np.float32).reshape(-1, 12))
    out = np.zeros(16, np.float64)
    L.orc_measure_disk(p, len(p), variant, G, remnant_frac, link_factor, roche, rho_fallback, pe_floor, pe_soft, out)
    return dict(zip(MEASURE_KEYS, out.tolist()))


# ---- relaxed-body assembly (gpu_sph.rs:260-339) ---------------------------------------------------------
def body_bulk(particles, prov: int):
    """body_bulk: (centre[3], mass, radius) of the particles with this provenance."""
    L = lib()
    L.orc_body_bulk.argtypes = [f32p, C.c_int, C.c_uint32, f64p]
    p = np.ascontiguousarray(np.ascontiguousarray(particles).view(np.float32).reshape(-1, 12))
    out = np.zeros(5, np.float64)
    L.orc_body_bulk(p, len(p), prov, out)
    return out[:3], float(out[3]), float(out[4])


def assemble(particles, placements):
    """assemble_from_relaxed_n: (particles, softening, dt); placements = [(offset, vel, spin), ...]."""
    L = lib()
    L.orc_assemble.argtypes = [f32p, C.c_int, f64p, C.c_int, f32p, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.orc_assemble.restype = C.c_int
    src = np.ascontiguousarray(particles)
    p = np.ascontiguousarray(src.view(np.float32).reshape(-1, 12))
    pl = np.ascontiguousarray(np.asarray(placements, np.float64).reshape(-1, 9))
    out = np.zeros_like(p)
    soft, dt = C.c_float(), C.c_float()
    m = L.orc_assemble(p, len(p), pl, len(pl), out, C.byref(soft), C.byref(dt))
    return out[:m].copy().view(src.dtype).reshape(-1), soft.value, dt.value


def dem_ground_step32(grains, prm, ground, heights=None, substeps=1):
    """The ground scene's substeps (contacts + integrate with cooling, drag, terrain, settle counter, glow) on a
    GRAIN_DTYPE array; ground = (center xyz, air_rho, drag_cd, specific_heat, cool_rate); heights[z, x] or None."""
    L = lib()
    i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    L.orc_dem_ground_step32.argtypes = [f32p, f32p, f32p, f32p, f32p, f32p, f32p, C.c_int, f32p, f32p,
                                        C.c_void_p, C.c_int, C.c_int]
    g = np.array(grains, copy=True)
    pos = np.ascontiguousarray(g["offset"], np.float32)
    vel = np.ascontiguousarray(g["vel"], np.float32)
    u = np.ascontiguousarray(g["u"], np.float32)
    rest = np.ascontiguousarray(g["resting"], np.float32)
    emis = np.ascontiguousarray(g["emission"], np.float32)
    rad = np.ascontiguousarray(g["radius"], np.float32)
    rho = np.ascontiguousarray(g["rho"], np.float32)
    gr = np.ascontiguousarray(ground, np.float32)
    if heights is None:
        hp, w, d = None, 0, 0
    else:
        h = np.ascontiguousarray(heights, np.int32)
        d, w = h.shape
        hp = h.ctypes.data_as(C.c_void_p)
    for _ in range(substeps):
        L.orc_dem_ground_step32(pos, vel, rad, rho, u, rest, emis, len(g), _c(prm, np.float32), gr, hp, w, d)
    g["offset"], g["vel"], g["u"], g["resting"], g["emission"] = pos, vel, u, rest, emis
    return g
