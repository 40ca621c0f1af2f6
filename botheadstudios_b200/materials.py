"""Tillotson material tables and the code-unit system.

The parameter values are the reference's catalogue entries (integrity-engine ``data/materials.json``:
basalt ``:155-166``, iron ``:520-531``; the same numbers as ``SphEos::basalt()/iron()`` in
``crates/engine/src/gpu_sph.rs:101-106``), kept in SI. A material row in the 48-byte exchange layout is
``[rho0, a, b, A, B, E0, E_iv, E_cv, alpha, beta, _p0, _p1]`` (``gpu_sph.rs:42``, ``sph_step.wgsl:43``).

Code units (G = 1, R_target = 1, M_target = 1): M_unit is the proto-Earth mass of the reference's body
catalogue (0.91 Earth masses), L_unit the radius of a 30 % iron / 70 % basalt-by-mass sphere of that mass at
the materials' reference densities, T_unit = sqrt(L³ / (G M)). The reference's SI-valued guards (the 1e-9
density floor, the 1 J/kg finite-difference floor of the sound speed, the 1e-9 m coincident-pair cut and the
1 m/s signal-speed floor, ``sph_step.wgsl:79,91,187,268``) are carried as explicit parameters and scaled.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

G_SI = 6.674e-11  # sph_step.wgsl:21, bh_gravity.wgsl:11, orbit::G

# name -> (rho0, a, b, A, B, E0, E_iv, E_cv, alpha, beta)
TILLOTSON_SI = {
    "basalt": (2700.0, 0.5, 1.5, 2.67e10, 2.67e10, 4.87e8, 4.72e6, 1.82e7, 5.0, 5.0),
    "iron": (7850.0, 0.5, 1.28, 1.28e11, 1.815e11, 1.425e7, 2.4e6, 8.67e6, 5.0, 5.0),
    # the catalogue's other layer materials, for the reference's layered bodies (HydroBody::particalize)
    "peridotite": (3500.0, 0.5, 1.4, 1.31e11, 4.9e10, 5.5e8, 4.5e6, 1.45e7, 5.0, 5.0),
    "ice": (917.0, 0.3, 0.1, 9.47e9, 9.47e9, 1.0e7, 7.73e5, 3.04e6, 10.0, 5.0),
}
# the catalogue's specific heats (J/kg/K), u = c·T for the layered bodies' geotherms
SPECIFIC_HEAT = {"basalt": 840.0, "iron": 449.0, "peridotite": 1000.0, "ice": 2090.0}
MAT_BASALT = 0  # gpu_sph.rs:107
MAT_IRON = 1  # gpu_sph.rs:108
MAT_PERIDOTITE = 2  # further rows of this library's material table (the engine's table holds up to 16)
MAT_ICE = 3
MAX_MATERIALS = 16  # gpu_sph.rs:113

EARTH_MASS = 5.972e24
PROTO_EARTH_MASS = 0.91 * EARTH_MASS


@dataclass(frozen=True)
class Units:
    """A unit system: lengths in L (m), masses in M (kg), times in T (s), with G = G_code."""

    L: float = 1.0
    M: float = 1.0
    T: float = 1.0
    G: float = G_SI

    @property
    def density(self):
        return self.M / self.L**3

    @property
    def pressure(self):
        return self.M / (self.L * self.T**2)

    @property
    def energy(self):  # specific energy, J/kg
        return self.L**2 / self.T**2

    @property
    def speed(self):
        return self.L / self.T

    # The reference's SI guards expressed in this unit system.
    @property
    def rho_floor(self):
        return 1.0e-9 / self.density

    @property
    def du_floor(self):
        return 1.0 / self.energy

    @property
    def r_min(self):
        return 1.0e-9 / self.L

    @property
    def sig_floor(self):
        return 1.0 / self.speed


SI = Units()


def code_units(total_mass_kg: float = PROTO_EARTH_MASS, iron_mass_frac: float = 0.3) -> Units:
    """G = 1 units where the target (30 % iron / 70 % basalt by mass) has M = 1 and R = 1."""
    rfe = TILLOTSON_SI["iron"][0]
    rba = TILLOTSON_SI["basalt"][0]
    vol = total_mass_kg * (iron_mass_frac / rfe + (1.0 - iron_mass_frac) / rba)
    L = (vol * 3.0 / (4.0 * math.pi)) ** (1.0 / 3.0)
    T = math.sqrt(L**3 / (G_SI * total_mass_kg))
    return Units(L=L, M=total_mass_kg, T=T, G=1.0)


def eos_row(name: str, units: Units = SI) -> np.ndarray:
    """One 12-float material row in the given units."""
    rho0, a, b, A, B, e0, eiv, ecv, al, be = TILLOTSON_SI[name]
    return np.array([rho0 / units.density, a, b, A / units.pressure, B / units.pressure, e0 / units.energy,
                     eiv / units.energy, ecv / units.energy, al, be, 0.0, 0.0], dtype=np.float32)


def eos_table(units: Units = SI, names=("basalt", "iron")) -> np.ndarray:
    """Material table [n_mat, 12] float32 (index = particle `mat`)."""
    return np.stack([eos_row(n, units) for n in names])


def eos_table64(units: Units = SI, names=("basalt", "iron")) -> np.ndarray:
    """The same table as f64 [n_mat, 10] (no padding), for the f64 physics."""
    out = []
    for n in names:
        rho0, a, b, A, B, e0, eiv, ecv, al, be = TILLOTSON_SI[n]
        out.append([rho0 / units.density, a, b, A / units.pressure, B / units.pressure, e0 / units.energy,
                    eiv / units.energy, ecv / units.energy, al, be])
    return np.array(out, dtype=np.float64)
