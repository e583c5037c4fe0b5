"""jw_average_and_symmetrize_noalloc, the symmetrisation for callers that
cannot allocate device memory (a program that gives all device memory to its
own pool allocator, or a time-critical loop that cannot afford cudaMalloc),
checked through the C ABI against the allocating jw_average_and_symmetrize on
two calls in a row.  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_symmetrize_matches_context_version():
    import torch
    import jimwlk as jw

    L = jw.lib()
    fn = L.jw_average_and_symmetrize_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    fn.restype = ctypes.c_int

    rng = np.random.default_rng(2024)
    for N in (64, 512):
        ctx = jw.Context(jw.config_defaults(Nx=N, Ny=N))
        f = ctx.field(1)
        buf = torch.empty((N, N, 2), dtype=torch.float64, device="cuda")
        for call in range(2):  # two calls in a row share the built-in scratch
            c = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
            f.set(c.reshape(N, N, 1))
            ctx.average_and_symmetrize(f)
            want = f.get()[..., 0]
            assert ctx.sync() == jw.OK
            buf.copy_(torch.from_numpy(np.stack([c.real, c.imag], axis=-1)))
            torch.cuda.synchronize()
            assert fn(ctypes.c_void_p(buf.data_ptr()), N, ctypes.c_void_p(0)) == jw.OK
            torch.cuda.synchronize()
            h = buf.cpu().numpy()
            got = h[..., 0] + 1j * h[..., 1]
            assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max(), (N, call)
        ctx.close()
    # beyond the built-in scratch: a clear error, nothing launched
    big = torch.zeros((1024, 1024, 2), dtype=torch.float64, device="cuda")
    assert fn(ctypes.c_void_p(big.data_ptr()), 1024, ctypes.c_void_p(0)) == jw.EINVAL
