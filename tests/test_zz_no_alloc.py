"""jw_average_and_symmetrize_noalloc, the symmetrisation for callers that
cannot allocate device memory (a program that gives all device memory to its
own pool allocator, or a time-critical loop that cannot afford cudaMalloc),
checked through the C ABI against the allocating jw_average_and_symmetrize on
two calls in a row.  Both run the same operations in the same order, so the
results agree bit for bit.  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fn():
    import jimwlk as jw
    fn = jw.lib().jw_average_and_symmetrize_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def test_noalloc_symmetrize_matches_context_version():
    import torch
    import jimwlk as jw

    fn = _fn()
    # set-up call: loads the device code and reserves the array, launches nothing
    assert fn(None, 0, None) == jw.OK
    rng = np.random.default_rng(2024)
    side = torch.cuda.Stream()
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
            # the second call runs on a stream of its own
            stream = side.cuda_stream if call == 1 else 0
            assert fn(ctypes.c_void_p(buf.data_ptr()), N, ctypes.c_void_p(stream)) == jw.OK
            torch.cuda.synchronize()
            h = buf.cpu().numpy()
            got = h[..., 0] + 1j * h[..., 1]
            assert np.array_equal(got, want), (N, call)
        ctx.close()


def test_noalloc_allocates_nothing_and_rejects_bad_input():
    import torch
    import jimwlk as jw

    fn = _fn()
    N = 256
    buf = torch.randn((N, N, 2), dtype=torch.float64, device="cuda")
    assert fn(ctypes.c_void_p(buf.data_ptr()), N, ctypes.c_void_p(0)) == jw.OK  # warm
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(3):
        assert fn(ctypes.c_void_p(buf.data_ptr()), N, ctypes.c_void_p(0)) == jw.OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0
    # beyond the built-in scratch, a misaligned array, no array: clear errors, nothing launched
    big = torch.zeros((1024, 1024, 2), dtype=torch.float64, device="cuda")
    assert fn(ctypes.c_void_p(big.data_ptr()), 1024, ctypes.c_void_p(0)) == jw.EINVAL
    assert fn(ctypes.c_void_p(buf.data_ptr() + 8), 16, ctypes.c_void_p(0)) == jw.EINVAL
    assert fn(None, 16, None) == jw.EINVAL
