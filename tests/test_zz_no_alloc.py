"""The allocation-free projection entry point against the handle-based one.

Some callers cannot allocate device memory: code running in a host callback, a hook
inside a framework whose caching allocator owns the GPU, or a real-time loop that may not
block on cudaMalloc.  ssfft_apply_projection_noalloc serves them with a fixed scratch
array compiled into the library; for the same input it must return what the
handle-based ssfft_apply_projection_device returns.  Collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _handle_projection(dims, mask, x):
    import torch

    from materialite_b200 import _native as nat
    from materialite_b200.engine import SolverHandle
    h = SolverHandle(dims, mask, "fp64")
    out = torch.empty_like(x)
    torch.cuda.synchronize()
    nat.check(h.lib.ssfft_apply_projection_device(h.h, ctypes.c_void_p(x.data_ptr()),
                                                  ctypes.c_void_p(out.data_ptr())))
    h.close()
    return out


def _noalloc_projection(dims, mask, x):
    import torch

    from materialite_b200 import _native as nat
    lib = nat.load_library()
    out = torch.empty_like(x)
    n = (ctypes.c_int32 * 3)(*dims)
    m = (ctypes.c_double * 6)(*mask)
    torch.cuda.synchronize()
    nat.check(lib.ssfft_apply_projection_noalloc(n, m, ctypes.c_void_p(x.data_ptr()),
                                                 ctypes.c_void_p(out.data_ptr()), None))
    return out


def test_noalloc_projection_matches_handle_entry_point():
    import torch
    cases = [((16, 12, 10), [0, 1, 1, 1, 1, 1], 1),
             ((32, 32, 32), [1, 1, 1, 1, 1, 1], 2),
             ((16, 12, 10), [0, 1, 1, 1, 1, 1], 1)]  # repeat: the shared array's old contents must not leak
    results = []
    for dims, mask, seed in cases:
        V = int(np.prod(dims))
        g = torch.Generator(device="cuda").manual_seed(seed)
        x = torch.randn(6, V, dtype=torch.float64, device="cuda", generator=g)
        got = _noalloc_projection(dims, mask, x)
        ref = _handle_projection(dims, mask, x)
        err = float((got - ref).norm() / ref.norm())
        assert err < 1e-12, (dims, err)
        results.append(got)
    assert torch.equal(results[0], results[2])


def test_noalloc_projection_rejects_oversized_grid():
    import torch

    from materialite_b200 import _native as nat
    lib = nat.load_library()
    dims = (80, 80, 80)  # beyond the 64^3 limit of the fixed scratch array
    x = torch.zeros(6, 16, dtype=torch.float64, device="cuda")
    n = (ctypes.c_int32 * 3)(*dims)
    m = (ctypes.c_double * 6)(*[0.0] * 6)
    rc = lib.ssfft_apply_projection_noalloc(n, m, ctypes.c_void_p(x.data_ptr()),
                                            ctypes.c_void_p(x.data_ptr()), None)
    assert rc == -4
    assert b"64^3" in lib.ssfft_last_error()
