"""The allocation-free tree gravity entry point (sph_gravity_tree_noalloc) against the context entry point.

Callers such as a real-time frame loop or an engine that owns all device memory cannot allocate when they need
forces; this entry point works out of a fixed array compiled into the library. The test passes device buffers
it allocated itself and compares two calls in a row (different point sets, so no state may leak from one call
into the next) with sph_gravity, which runs the same walk with its own allocations.
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


@pytest.mark.parametrize("leaf,quad", [(16, 1), (8, 0)])
def test_noalloc_tree_gravity_matches_context_entry_point_twice(leaf, quad):
    import torch

    L = _lib.load()
    for call, (n, seed) in enumerate(((20000, 21), (4096, 22))):
        _, pos, mass = cloud(n, seed)
        with GpuSph(n, G=G, theta=0.5, leaf_size=leaf, multipole=quad) as s:
            ref = s.gravity(pos, mass, SOFT, "tree")
        bodies = torch.tensor(np.concatenate([pos, mass[:, None]], axis=1).astype(np.float32), device="cuda:0")
        out = torch.full((n, 4), float("nan"), dtype=torch.float32, device="cuda:0")
        stream = torch.cuda.current_stream(0)
        st = L.sph_gravity_tree_noalloc(C.c_void_p(bodies.data_ptr()), n, G, SOFT, 0.5, leaf, quad,
                                        C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == _lib.SPH_OK, (call, st)
        stream.synchronize()
        a = out[:, :3].double().cpu().numpy()
        assert np.isfinite(a).all()
        rms = np.sqrt(((a - ref) ** 2).sum() / (ref ** 2).sum())
        rel = np.linalg.norm(a - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert rms < 1e-6 and rel.max() < 1e-5, (call, rms, rel.max())


def test_noalloc_rejects_sizes_beyond_its_array():
    L = _lib.load()
    fake = C.c_void_p(1)  # never dereferenced: the size check comes first
    assert L.sph_gravity_tree_noalloc(fake, 65537, G, SOFT, 0.5, 16, 1, fake, None) == _lib.SPH_ERR_INVALID
    assert L.sph_gravity_tree_noalloc(fake, 1000, G, SOFT, 0.5, 4, 1, fake, None) == _lib.SPH_ERR_INVALID
