"""Host-side mirror of the engine's granular pipeline ``GpuParticles`` (crates/engine/src/gpu_particles.rs:46-325)
over the C ABI: ``new``/``replace``/``set_params``/``dispatch``/``readback``/``count``, plus the ground scene's
medium and terrain (``set_ground``, ``set_terrain``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import GRAIN_DTYPE, DemGround, DemParams
from .gpusph import SphError


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class GpuGrains:
    def __init__(self, capacity: int, device: int = -1):
        self._L = _lib.load()
        h = C.c_void_p()
        st = self._L.sph_dem_create(int(capacity), int(device), C.byref(h))
        if st != 0:
            raise SphError(st, "sph_dem_create failed")
        self._h = h

    def _check(self, st, what):
        if st < 0:
            raise SphError(st, what)
        return st

    def set_params(self, dt, stiffness, normal_damp, friction, tangent_damp, cohesion=0.0, gravity=(0.0, -9.81, 0.0)):
        p = DemParams()
        p.gravity[:] = gravity
        p.dt, p.c_stiffness, p.c_normal_damp = dt, stiffness, normal_damp
        p.c_friction, p.c_tangent_damp, p.c_cohesion = friction, tangent_damp, cohesion
        self._check(self._L.sph_dem_set_params(self._h, C.byref(p)), "sph_dem_set_params")

    def set_ground(self, center=(0.0, 0.0, 0.0), air_rho=0.0, drag_cd=0.0, specific_heat=0.0, cool_rate=0.0):
        """The scene's heightfield frame, air (drag) and thermal relaxation (particle_step.wgsl Params)."""
        g = DemGround()
        g.center[:] = center
        g.air_rho, g.drag_cd, g.specific_heat, g.cool_rate = air_rho, drag_cd, specific_heat, cool_rate
        self._check(self._L.sph_dem_set_ground(self._h, C.byref(g)), "sph_dem_set_ground")

    def set_terrain(self, heights):
        """heights[z, x]: column tops in voxel units (None removes the terrain)."""
        if heights is None:
            self._check(self._L.sph_dem_set_terrain(self._h, None, 0, 0), "sph_dem_set_terrain")
            return
        h = np.ascontiguousarray(heights, dtype=np.int32)
        d, w = h.shape
        self._check(self._L.sph_dem_set_terrain(self._h, _ptr(h), w, d), "sph_dem_set_terrain")

    def replace(self, grains: np.ndarray) -> int:
        g = np.ascontiguousarray(grains, dtype=GRAIN_DTYPE)
        return self._check(self._L.sph_dem_replace(self._h, _ptr(g), len(g)), "sph_dem_replace")

    def dispatch(self, substeps: int = 1):
        self._check(self._L.sph_dem_step(self._h, int(substeps)), "sph_dem_step")

    def readback(self) -> np.ndarray:
        out = np.zeros(max(self.count(), 1), GRAIN_DTYPE)
        n = C.c_uint32()
        self._check(self._L.sph_dem_readback(self._h, _ptr(out), len(out), C.byref(n)), "sph_dem_readback")
        return out[: n.value]

    def contacts(self) -> np.ndarray:
        out = np.zeros((self.count(), 16), np.float32)
        self._check(self._L.sph_dem_contacts(self._h, _ptr(out), out.nbytes), "sph_dem_contacts")
        return out

    def count(self) -> int:
        return int(self._L.sph_dem_count(self._h))

    def close(self):
        if getattr(self, "_h", None):
            self._L.sph_dem_destroy(self._h)
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


def grain_pack(n: int, radius: float = 0.5, spacing: float = 0.97, jitter: float = 0.02, seed: int = 0,
               vel_scale: float = 0.3) -> np.ndarray:
    """A seeded, slightly overlapping cubic pack of equal grains (a settling pile) with random velocities."""
    rng = np.random.default_rng(seed)
    m = int(np.ceil(n ** (1.0 / 3.0)))
    idx = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)[:n]
    g = np.zeros(n, GRAIN_DTYPE)
    g["offset"] = idx * (2.0 * radius * spacing) + rng.uniform(-jitter, jitter, (n, 3))
    g["vel"] = rng.uniform(-vel_scale, vel_scale, (n, 3))
    g["radius"] = radius
    g["rho"] = 2700.0
    return g
