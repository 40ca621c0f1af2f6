"""The allocation-free tree gravity entry point (sph_gravity_tree_noalloc) against the context entry point.

Callers such as a real-time frame loop or an engine that owns all device memory cannot allocate when they need
forces; this entry point works out of a fixed array compiled into the library. The test passes device buffers
it allocated itself and compares two calls in a row (different point sets, so no state may leak from one call
into the next) with sph_gravity, which runs the same walk with its own allocations. It also runs the largest
case the array holds (65,536 points in 8-point leaves, which fills the node arrays exactly) and checks the
potential in .w against an FP64 direct sum.
This file is collected last on purpose and also passes when run on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from botheadstudios_b200 import _lib
from botheadstudios_b200.gpusph import GpuSph
from refcases import cloud

pytestmark = pytest.mark.gpu
G = 6.674e-11
SOFT = 5.0e3


def _noalloc(pos, mass, leaf, quad, theta=0.5):
    import torch

    L = _lib.load()
    n = len(mass)
    bodies = torch.tensor(np.concatenate([pos, mass[:, None]], axis=1).astype(np.float32), device="cuda:0")
    out = torch.full((n, 4), float("nan"), dtype=torch.float32, device="cuda:0")
    stream = torch.cuda.current_stream(0)
    st = L.sph_gravity_tree_noalloc(C.c_void_p(bodies.data_ptr()), n, G, SOFT, theta, leaf, quad,
                                    C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert st == _lib.SPH_OK, st
    stream.synchronize()
    return out.double().cpu().numpy()


def _close_to_context(pos, mass, leaf, quad, theta=0.5):
    with GpuSph(len(mass), G=G, theta=theta, leaf_size=leaf, multipole=quad) as s:
        ref = s.gravity(pos, mass, SOFT, "tree")
    a = _noalloc(pos, mass, leaf, quad, theta)[:, :3]
    assert np.isfinite(a).all()
    rms = np.sqrt(((a - ref) ** 2).sum() / (ref ** 2).sum())
    rel = np.linalg.norm(a - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert rms < 1e-6 and rel.max() < 1e-5, (len(mass), rms, rel.max())


@pytest.mark.parametrize("leaf,quad", [(16, 1), (8, 0)])
def test_noalloc_tree_gravity_matches_context_entry_point_twice(leaf, quad):
    for n, seed in ((20000, 21), (4096, 22)):
        _, pos, mass = cloud(n, seed)
        _close_to_context(pos, mass, leaf, quad)


def test_noalloc_largest_case_fills_the_array():
    """65,536 points in 8-point leaves: the node arrays' full size (2·8192 − 1 nodes)."""
    _, pos, mass = cloud(65536, 23)
    _close_to_context(pos, mass, 8, 1)


def test_noalloc_potential_against_fp64_direct_sum():
    n = 4096
    _, pos, mass = cloud(n, 24)
    phi = _noalloc(pos, mass, 8, 1, theta=0.3)[:, 3]
    ref = np.zeros(n)
    for a in range(0, n, 512):
        d = pos[a:a + 512, None, :] - pos[None, :, :]
        r = np.sqrt((d * d).sum(-1) + SOFT * SOFT)
        inv = mass[None, :] / r
        inv[np.arange(min(512, n - a)), np.arange(a, min(a + 512, n))] = 0.0  # no self term
        ref[a:a + 512] = -G * inv.sum(1)
    rel = np.abs(phi - ref) / np.abs(ref)
    assert np.isfinite(phi).all() and rel.max() < 1e-3, rel.max()


def test_noalloc_rejects_sizes_beyond_its_array_and_misaligned_buffers():
    L = _lib.load()
    fake = C.c_void_p(256)  # never dereferenced: the argument checks come first
    assert L.sph_gravity_tree_noalloc(fake, 65537, G, SOFT, 0.5, 16, 1, fake, None) == _lib.SPH_ERR_INVALID
    assert L.sph_gravity_tree_noalloc(fake, 1000, G, SOFT, 0.5, 4, 1, fake, None) == _lib.SPH_ERR_INVALID
    odd = C.c_void_p(256 + 4)
    assert L.sph_gravity_tree_noalloc(odd, 1000, G, SOFT, 0.5, 16, 1, fake, None) == _lib.SPH_ERR_INVALID
    assert L.sph_gravity_tree_noalloc(fake, 1000, G, SOFT, 0.5, 16, 1, odd, None) == _lib.SPH_ERR_INVALID
