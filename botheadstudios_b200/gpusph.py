"""Host-side mirror of the engine's ``GpuSph`` (crates/engine/src/gpu_sph.rs:742-922) over the C ABI.

Method names follow the reference: ``new``/``upload``/``set_dt``/``set_av``/``encode_relax``/``encode_kdk``/
``begin_readback``/``take_readback``/``particle_buffer``/``count``. As in the reference, ``upload`` clamps
to capacity, ``encode_*`` only enqueue work, and ``take_readback`` returns ``None`` until the two-phase
readback has landed. Device-side failures raise :class:`SphError` (the reference has no error path there;
this one does not hide them).
"""
from __future__ import annotations

import ctypes as C
import warnings
from typing import Optional

import numpy as np

from . import _lib
from ._lib import PARTICLE_DTYPE, Q, SphDiag


class SphError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class GpuSph:
    """A B200 SPH solver context (one CUDA stream, device-resident state)."""

    def __init__(self, capacity: int, config=None, **cfg):
        self._L = _lib.load()
        self.config = config if config is not None else _lib.default_config(**cfg)
        h = C.c_void_p()
        st = self._L.sph_create(C.byref(self.config), int(capacity), C.byref(h))
        if st != 0:
            raise SphError(st, "sph_create failed: " + self._L.sph_status_string(st).decode())
        self._h = h
        self.capacity = int(capacity)
        self.softening = 0.0

    @classmethod
    def new(cls, capacity: int, **cfg) -> "GpuSph":
        return cls(capacity, **cfg)

    # ---- error handling ------------------------------------------------------------------------------
    def _check(self, st: int, what: str) -> int:
        if st < 0:
            raise SphError(st, f"{what}: {self._L.sph_last_error(self._h).decode()}"
                               f" [{self._L.sph_status_string(st).decode()}]")
        return st

    # ---- GpuSph surface ------------------------------------------------------------------------------
    def upload(self, particles: np.ndarray, eos: np.ndarray, softening: float) -> int:
        p = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        e = np.ascontiguousarray(eos, dtype=np.float32).reshape(-1, 12)
        st = self._check(self._L.sph_upload(self._h, _ptr(p), len(p), _ptr(e), len(e), float(softening)),
                         "sph_upload")
        if st == _lib.SPH_CLAMPED:
            warnings.warn("upload clamped to capacity / material table size")
        self.softening = float(softening)
        self.n_impacts = 1
        return st

    def upload_batch(self, particles: np.ndarray, offsets, eos: np.ndarray, softening) -> int:
        """Independent impacts in one context: impact k = particles[offsets[k]:offsets[k+1]], each with its
        own softening (a scalar applies to all). Every phase of a step is one launch over all impacts."""
        p = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        off = np.ascontiguousarray(offsets, dtype=np.uint32)
        k = len(off) - 1
        soft = np.ascontiguousarray(np.broadcast_to(np.asarray(softening, np.float32), (k,)))
        e = np.ascontiguousarray(eos, dtype=np.float32).reshape(-1, 12)
        if k < 1 or int(off[-1]) != len(p):
            raise ValueError("offsets must start at 0 and end at len(particles)")
        st = self._check(self._L.sph_upload_batch(self._h, _ptr(p), _ptr(off), k, _ptr(e), len(e), _ptr(soft)),
                         "sph_upload_batch")
        self.n_impacts = k
        self.softening = soft.copy()
        return st

    def impact_dt(self) -> np.ndarray:
        """dt of each impact's last step."""
        out = np.zeros(getattr(self, "n_impacts", 1), np.float64)
        self._check(self._L.sph_inspect(self._h, Q["IMPACT_DT"], _ptr(out), out.nbytes), "sph_inspect(IMPACT_DT)")
        return out

    def impact_time(self) -> np.ndarray:
        """Simulated time of each impact."""
        out = np.zeros(getattr(self, "n_impacts", 1), np.float64)
        self._check(self._L.sph_inspect(self._h, Q["IMPACT_TIME"], _ptr(out), out.nbytes),
                    "sph_inspect(IMPACT_TIME)")
        return out

    # ---- relaxed-body assembly --------------------------------------------------------------------------
    def body_bulk(self, prov: int):
        """body_bulk on the device: (centre[3], mass, 98 %-mass radius) of the particles with this provenance."""
        c = (C.c_double * 3)()
        m, r = C.c_double(), C.c_double()
        self._check(self._L.sph_body_bulk(self._h, prov, c, C.byref(m), C.byref(r)), "sph_body_bulk")
        return np.array(c[:], np.float64), m.value, r.value

    def assemble(self, placements):
        """assemble_from_relaxed_n on the device: placements[k] = (offset, vel, spin) for source body prov = k.
        The state becomes the assembled impact; returns (softening, dt) as the reference does."""
        arr = (_lib.Placement * max(len(placements), 1))()
        for k, (o, v, w) in enumerate(placements):
            arr[k].offset[:] = [float(x) for x in o]
            arr[k].vel[:] = [float(x) for x in v]
            arr[k].spin[:] = [float(x) for x in w]
        soft, dt = C.c_float(), C.c_float()
        self._check(self._L.sph_assemble(self._h, arr, len(placements), C.byref(soft), C.byref(dt)), "sph_assemble")
        self.softening = soft.value
        self.n_impacts = 1
        return soft.value, dt.value

    # ---- disk measurement ----------------------------------------------------------------------------
    def measure_disk(self, impact: int = 0, variant: int = 0, **kw) -> dict:
        """Disk measurement and Moon candidate of one impact on the device (sph_measure_disk). variant 0 is the
        impact-run tool's `measure`, 1 the engine's disk statistics; keyword arguments override the
        sph_measure_cfg defaults (G, remnant_frac, link_factor, roche, rho_fallback, pe_floor, pe_softening)."""
        cfg = _lib.MeasureCfg()
        self._L.sph_measure_default(C.byref(cfg))
        cfg.variant = variant
        for k, v in kw.items():
            if not hasattr(cfg, k):
                raise TypeError(f"unknown measure option {k}")
            setattr(cfg, k, v)
        out = _lib.DiskMeasure()
        self._check(self._L.sph_measure_disk(self._h, impact, C.byref(cfg), C.byref(out)), "sph_measure_disk")
        return {name: getattr(out, name) for name, _ in out._fields_}

    # ---- learned smoothing lengths --------------------------------------------------------------------
    def mlp_set(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self._L.sph_mlp_set(self._h, _ptr(p), len(p)), "sph_mlp_set")

    def mlp_record(self, on: bool = True):
        self._check(self._L.sph_mlp_record(self._h, 1 if on else 0), "sph_mlp_record")

    def mlp_features(self):
        """(features[n][8], Δlog h[n]) of the last recorded step, in original particle order."""
        n = self.count()
        f = np.zeros((n, 8), np.float32)
        d = np.zeros(n, np.float32)
        self._check(self._L.sph_mlp_features(self._h, _ptr(f), _ptr(d), n), "sph_mlp_features")
        return f, d

    def set_progress(self, fraction: float):
        self._check(self._L.sph_set_progress(self._h, float(fraction)), "sph_set_progress")

    def set_dt(self, dt: float, damp: float = 1.0):
        self._check(self._L.sph_set_dt(self._h, float(dt), float(damp)), "sph_set_dt")

    def set_av(self, alpha: float, beta: float):
        self._check(self._L.sph_set_av(self._h, float(alpha), float(beta)), "sph_set_av")

    def set_omega(self, omega: float):
        self._check(self._L.sph_set_omega(self._h, float(omega)), "sph_set_omega")

    def encode_kdk(self, substeps: int):
        self._check(self._L.sph_step_kdk(self._h, int(substeps)), "sph_step_kdk")

    def encode_relax(self, steps: int):
        self._check(self._L.sph_step_relax(self._h, int(steps)), "sph_step_relax")

    def eval_forces(self):
        self._check(self._L.sph_eval_forces(self._h), "sph_eval_forces")

    def begin_readback(self):
        self._check(self._L.sph_readback_begin(self._h), "sph_readback_begin")

    def take_readback(self) -> Optional[np.ndarray]:
        out = np.empty(max(self.count(), 1), dtype=PARTICLE_DTYPE)
        n = C.c_uint32()
        ready = C.c_int()
        st = self._L.sph_readback_take(self._h, _ptr(out), len(out), C.byref(n), C.byref(ready))
        if st == _lib.SPH_NOT_READY:
            return None
        self._check(st, "sph_readback_take")
        return out[: n.value]

    def readback_into(self, out: np.ndarray) -> int:
        """Blocking readback straight into `out` (a PARTICLE_DTYPE array, ideally in pinned memory)."""
        assert out.dtype == PARTICLE_DTYPE and out.flags["C_CONTIGUOUS"]
        n = C.c_uint32()
        self._check(self._L.sph_readback_into(self._h, _ptr(out), len(out), C.byref(n)), "sph_readback_into")
        return int(n.value)

    def readback(self) -> np.ndarray:
        """Blocking convenience: begin, sync, take."""
        self.begin_readback()
        self.sync()
        r = self.take_readback()
        assert r is not None
        return r

    def count(self) -> int:
        return int(self._L.sph_count(self._h))

    def particle_buffer(self) -> int:
        p = C.c_void_p()
        self._check(self._L.sph_particle_buffer(self._h, C.byref(p)), "sph_particle_buffer")
        return int(p.value or 0)

    def sync(self, timeout_ms: int = 0):
        self._check(self._L.sph_sync(self._h, int(timeout_ms)), "sph_sync")

    def stream(self) -> int:
        return int(self._L.sph_stream(self._h) or 0)

    def diag(self, check: bool = True) -> dict:
        d = SphDiag()
        st = self._L.sph_diag(self._h, C.byref(d))
        if check:
            self._check(st, "sph_diag")
        return dict(kinetic=d.kinetic, internal=d.internal, potential=d.potential, momentum=list(d.momentum),
                    angular_momentum=list(d.angular_momentum), mass=d.mass, dt=d.dt, time=d.time, steps=d.steps,
                    max_neighbours_seen=d.max_neighbours_seen, overflow_flags=d.overflow_flags,
                    h_iterations=d.h_iterations, h_residual=d.h_residual, h_accepted=d.h_accepted,
                    walk_nodes=d.walk_nodes,
                    walk_pops=d.walk_pops, m2p_interactions=d.m2p_interactions,
                    p2p_interactions=d.p2p_interactions, local_expansions=d.local_expansions,
                    p2p_slots=d.p2p_slots, status=st)

    # ---- profiling ------------------------------------------------------------------------------------
    def profile_enable(self, on: bool = True):
        self._check(self._L.sph_profile_enable(self._h, int(on)), "sph_profile_enable")

    def profile_read(self) -> dict:
        pr = _lib.SphProfile()
        self._check(self._L.sph_profile_read(self._h, C.byref(pr)), "sph_profile_read")
        return dict(ms={k: pr.ms[i] for i, k in enumerate(_lib.PHASES)},
                    calls={k: int(pr.calls[i]) for i, k in enumerate(_lib.PHASES)},
                    kernel_launches=int(pr.kernel_launches))

    # ---- inspection / gravity ------------------------------------------------------------------------
    def inspect(self, what: str) -> np.ndarray:
        n = self.count()
        L = self.n_leaves()
        nn = max(2 * L - 1, 0)
        cap = int(self.config.max_neighbours)
        k = getattr(self, "n_impacts", 1)
        shapes = dict(BBOX=(np.float32, (6,) if k == 1 else (k, 6)), CODES=(np.uint32, (n,)), ORDER=(np.uint32, (n,)),
                      LEFT=(np.uint32, (max(L - 1, 0),)), RIGHT=(np.uint32, (max(L - 1, 0),)),
                      PARENT=(np.uint32, (nn,)), NODE_COM=(np.float32, (nn, 4)), NODE_BMIN=(np.float32, (nn, 4)),
                      NODE_BMAX=(np.float32, (nn, 4)), NBR_COUNT=(np.uint32, (n,)), NBR_LIST=(np.uint32, (n, cap)),
                      RHO=(np.float32, (n,)), PRESSURE=(np.float32, (n,)), SOUND=(np.float32, (n,)),
                      ACC_SPH=(np.float32, (n, 4)), ACC_GRAV=(np.float32, (n, 4)), H=(np.float32, (n,)))
        dt, shape = shapes[what]
        out = np.zeros(shape, dtype=dt)
        if out.nbytes == 0:
            return out
        self._check(self._L.sph_inspect(self._h, Q[what], _ptr(out), out.nbytes), f"sph_inspect({what})")
        return out

    def n_leaves(self) -> int:
        v = np.zeros(1, np.uint32)
        self._check(self._L.sph_inspect(self._h, Q["N_LEAVES"], _ptr(v), 4), "sph_inspect(N_LEAVES)")
        return int(v[0])

    def neighbour_sets(self):
        cnt = self.inspect("NBR_COUNT")
        lst = self.inspect("NBR_LIST")
        return [np.sort(lst[i, : cnt[i]]) for i in range(len(cnt))]

    def gravity(self, pos3, mass, softening: float, mode: str = "tree") -> np.ndarray:
        p = np.ascontiguousarray(pos3, dtype=np.float64)
        m = np.ascontiguousarray(mass, dtype=np.float64)
        acc = np.zeros((len(m), 3), np.float64)
        self._check(self._L.sph_gravity(self._h, _ptr(p), _ptr(m), len(m), float(softening),
                                        _lib.GRAVITY[mode], _ptr(acc)), "sph_gravity")
        return acc

    def gravity_direct64(self, pos3, mass, softening: float, targets=None) -> np.ndarray:
        p = np.ascontiguousarray(pos3, dtype=np.float64)
        m = np.ascontiguousarray(mass, dtype=np.float64)
        if targets is None:
            tp, nt = None, len(m)
        else:
            t = np.ascontiguousarray(targets, dtype=np.uint32)
            tp, nt = _ptr(t), len(t)
        acc = np.zeros((nt, 3), np.float64)
        self._check(self._L.sph_gravity_direct64(self._h, _ptr(p), _ptr(m), len(m), tp, nt, float(softening),
                                                 _ptr(acc)), "sph_gravity_direct64")
        return acc

    def close(self):
        if getattr(self, "_h", None):
            self._L.sph_destroy(self._h)
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


def particles_from_arrays(pos, h, vel, u, mass, mat, rho=None, prov=None) -> np.ndarray:
    """Pack SoA arrays into the 48-byte exchange layout."""
    n = len(mass)
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    p["pos"] = pos
    p["h"] = h
    p["vel"] = vel
    p["u"] = u
    p["mass"] = mass
    p["mat"] = mat
    p["rho"] = 0.0 if rho is None else rho
    p["prov"] = 0 if prov is None else prov
    return p
