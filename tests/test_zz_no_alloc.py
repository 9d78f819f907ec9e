"""The allocation-free entry point pgm_field_static against pgm_field (GPU).

pgm_field_static exists for callers that cannot allocate device memory (a jax.ffi custom call inside
XLA, which owns the GPU's memory and hands the call its buffers; code recording a CUDA graph).  It
keeps its intermediates in one static device array shared by all calls, so two calls in a row must
each give the result of the handle-based pgm_field: the second call sees the first one's leftovers
and must clear what it accumulates into.  This file is collected last, so a run that stops at the
first failure has already run every other test; it also passes alone in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

# the tolerance of the FP64 field tests of test_gpu_parity.py
TOL = 1e-10


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_static_field_equals_handle_field_twice():
    from conftest import SMALL_BOX_SETTINGS

    from pgm_jax_b200 import _lib
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.systems import small_box

    s, pos, H = small_box(0)
    st = dict(SMALL_BOX_SETTINGS)
    ff = PGMForceField(s, H, MDSettings(precision="double", **st))
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    f64 = lambda a: torch.tensor(np.ascontiguousarray(a, float), dtype=torch.float64, device=dev)  # noqa: E731
    x, box, q, rad = f64(pos), f64(H), f64(s.q), f64(s.radius)
    grid_c = (C.c_int * 3)(*st["pme_grid"])
    rng = np.random.default_rng(11)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    for call, charges in enumerate((True, False)):
        d_np = rng.normal(scale=0.01, size=(s.n, 3))
        d = f64(d_np)
        ref = ff.field(pos, H, d_np, charges=charges).cpu().numpy()
        out = torch.full((s.n, 3), np.nan, dtype=torch.float64, device=dev)
        rc = lib.pgm_field_static(stream, s.n, _p(x), _p(box), _p(q), _p(rad), st["cutoff"], st["ewald_beta"], grid_c,
                                  st["pme_order"], int(charges), _p(d), _p(out))
        assert rc == 0, lib.pgm_static_last_error().decode()
        got = out.cpu().numpy()
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err <= TOL, (call, err)


def test_static_field_rejects_oversized_inputs():
    from pgm_jax_b200 import _lib

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    z = torch.zeros((8, 3), dtype=torch.float64, device=dev)
    box = torch.eye(3, dtype=torch.float64, device=dev)
    r = torch.full((8,), 0.05, dtype=torch.float64, device=dev)
    grid_c = (C.c_int * 3)(128, 128, 128)
    rc = lib.pgm_field_static(None, 8, _p(z), _p(box), _p(r), _p(r), 0.4, 6.0, grid_c, 6, 1, _p(z), _p(z))
    assert rc == 4 and b"mesh" in lib.pgm_static_last_error()
    grid_c = (C.c_int * 3)(16, 16, 16)
    rc = lib.pgm_field_static(None, 5000, _p(z), _p(box), _p(r), _p(r), 0.4, 6.0, grid_c, 6, 1, _p(z), _p(z))
    assert rc == 4 and b"n_atoms" in lib.pgm_static_last_error()


def test_static_field_box_too_small_for_the_cutoff_gives_nan():
    """A box whose half height is below the cutoff cannot be served by the minimum image: the
    field is NaN (not a silently wrong value), and the next valid call is correct again."""
    from pgm_jax_b200 import _lib
    from pgm_jax_b200.systems import small_box

    s, pos, H = small_box(0)
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    f64 = lambda a: torch.tensor(np.ascontiguousarray(a, float), dtype=torch.float64, device=dev)  # noqa: E731
    x, box, q, rad = f64(pos), f64(H), f64(s.q), f64(s.radius)
    d = f64(np.random.default_rng(2).normal(scale=0.01, size=(s.n, 3)))
    grid_c = (C.c_int * 3)(32, 32, 32)
    out = torch.zeros((s.n, 3), dtype=torch.float64, device=dev)
    cutoff = 0.6 * float(np.min(np.diag(H)))  # above half the smallest diagonal element
    rc = lib.pgm_field_static(None, s.n, _p(x), _p(box), _p(q), _p(rad), cutoff, 6.0, grid_c, 6, 1, _p(d), _p(out))
    assert rc == 0, lib.pgm_static_last_error().decode()
    assert torch.isnan(out).all()
    rc = lib.pgm_field_static(None, s.n, _p(x), _p(box), _p(q), _p(rad), 0.6, 6.0, grid_c, 6, 1, _p(d), _p(out))
    assert rc == 0 and torch.isfinite(out).all()
