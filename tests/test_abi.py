"""The C ABI boundary, checked without a GPU: the library exports every symbol the header declares, and the
ctypes mirror has the header's struct layouts (the reference pins its repr(C) structs to the WGSL ones the
same way, crates/engine/src/gpu_sph.rs:937-996)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from botheadstudios_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sph_b200.h")


@pytest.fixture(scope="module")
def libpath():
    return build.build()


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sph_[a-z0-9_]+)\s*\(", src)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(libpath):
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (sph_[a-z0-9_]+)", out))
    missing = set(declared_functions()) - exported
    assert not missing, missing


def test_library_loads_without_gpu(libpath):
    L = _lib.load()
    for name in _lib.EXPORTS:
        assert hasattr(L, name)
    assert L.sph_status_string(-5).decode() == "device capacity overflow"
    cfg = _lib.default_config()
    assert cfg.G == pytest.approx(6.674e-11) and cfg.theta == pytest.approx(0.5) and cfg.leaf_size == 1


def test_struct_layouts_match_header():
    prog = r"""
#include <stdio.h>
#include <stddef.h>
#include "sph_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(SphParticle48), sizeof(SphEos48), sizeof(sph_config), sizeof(sph_diag_out));
  printf("%zu %zu %zu %zu %zu %zu\n", offsetof(SphParticle48, h), offsetof(SphParticle48, vel),
         offsetof(SphParticle48, u), offsetof(SphParticle48, mat), offsetof(SphParticle48, rho),
         offsetof(SphParticle48, prov));
  printf("%zu %zu %zu %zu %zu %zu\n", offsetof(sph_config, theta), offsetof(sph_config, max_neighbours),
         offsetof(sph_config, cfl), offsetof(sph_config, sig_floor), offsetof(sph_config, walk_stack),
         offsetof(sph_config, local_theta));
  printf("%zu %zu %zu\n", offsetof(sph_diag_out, dt), offsetof(sph_diag_out, steps),
         offsetof(sph_diag_out, h_residual));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        open(c, "w").write(prog)
        exe = os.path.join(d, "l")
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = list(map(int, lines[0].split()))
    assert sizes == [48, 48, C.sizeof(_lib.SphConfig), C.sizeof(_lib.SphDiag)]
    p = _lib.PARTICLE_DTYPE
    assert list(map(int, lines[1].split())) == [p.fields[k][1] for k in ("h", "vel", "u", "mat", "rho", "prov")]
    sc = _lib.SphConfig
    assert list(map(int, lines[2].split())) == [sc.theta.offset, sc.max_neighbours.offset, sc.cfl.offset,
                                                sc.sig_floor.offset, sc.walk_stack.offset, sc.local_theta.offset]
    sd = _lib.SphDiag
    assert list(map(int, lines[3].split())) == [sd.dt.offset, sd.steps.offset, sd.h_residual.offset]


def test_ic_generator_counts_and_composition():
    from botheadstudios_b200 import ic
    I = ic.impact(8192, 2048)
    p = I.particles
    assert len(p) == 10240 and p.dtype.itemsize == 48
    assert np.isclose(p["mass"][:8192].sum(), 1.0, rtol=1e-5) and np.isclose(p["mass"][8192:].sum(), 0.1, rtol=1e-5)
    iron = p["mat"] == 1
    assert np.isclose(p["mass"][iron].sum() / p["mass"].sum(), 0.3, atol=1e-3)
    mom = (p["mass"][:, None].astype(np.float64) * p["vel"]).sum(0)
    assert np.abs(mom).max() < 1e-6
    r = np.linalg.norm(I.pos64[:8192] - I.pos64[:8192].mean(0), axis=1)
    assert 0.95 < r.max() < 1.1


def test_grain_layouts_match_header():
    prog = r"""
#include <stdio.h>
#include <stddef.h>
#include "sph_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(SphGrain80), offsetof(SphGrain80, radius), offsetof(SphGrain80, rho),
         sizeof(sph_dem_params), offsetof(sph_dem_params, dt), offsetof(sph_dem_params, c_cohesion));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "g.c")
        open(c, "w").write(prog)
        exe = os.path.join(d, "g")
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        vals = list(map(int, subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()))
    g = _lib.GRAIN_DTYPE
    assert vals == [80, g.fields["radius"][1], g.fields["rho"][1], C.sizeof(_lib.DemParams), _lib.DemParams.dt.offset,
                    _lib.DemParams.c_cohesion.offset]
