"""shm_rescale_noalloc: the rescale for callers that cannot allocate device
memory (a host whose own pool owns all device memory, a latency-critical path
that cannot take cudaMalloc's implicit synchronisation, an FFI caller without a
device allocator).  It must give exactly what shm_rescale gives (integer work:
bit for bit), on two calls in a row, allocate nothing while doing so (neither
the library's pool nor torch's caching allocator grows), accept an empty batch
without leaving an error behind, and refuse sizes beyond its fixed scratch.

This file is collected last so a failure here leaves every other test run."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BITS = [60] + [50] * 23 + [60] * 8  # N = 2^16, 24 + 8 primes


def _noalloc(lib, ctx, t_in, t_out, n_polys, L):
    import torch

    return lib.shm_rescale_noalloc(ctx._h, ctypes.c_void_p(t_in.data_ptr()), ctypes.c_void_p(t_out.data_ptr()),
                                   n_polys, L, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def _memory(lib, ctx):
    """(pool reserved, pool used, torch reserved, torch allocated) in bytes."""
    import torch

    torch.cuda.synchronize()
    reserved, used = ctypes.c_size_t(0), ctypes.c_size_t(0)
    assert lib.shm_pool_usage(ctx._h, ctypes.byref(reserved), ctypes.byref(used), None, 0) == 0
    return reserved.value, used.value, torch.cuda.memory_reserved(), torch.cuda.memory_allocated()


def test_rescale_noalloc_matches_rescale_on_two_calls():
    import torch

    from shmoai_b200._lib import lib
    from shmoai_b200.ckks import CKKSContext

    L = lib()
    L.shm_rescale_noalloc.restype = ctypes.c_int
    L.shm_rescale_noalloc.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_uint32] * 2 + [ctypes.c_void_p]
    L.shm_rescale_noalloc_max_words.restype = ctypes.c_size_t
    L.shm_pool_usage.restype = ctypes.c_int
    L.shm_pool_usage.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int]
    ctx = CKKSContext(16, bits=BITS, n_special=8)
    n, lv = ctx.n, ctx.nq
    assert L.shm_rescale_noalloc_max_words() * 8 == 32 << 20
    pr = torch.tensor(ctx.primes[:lv].astype(np.int64), device="cuda").view(1, lv, 1)
    g = torch.Generator(device="cuda").manual_seed(1)
    # inputs, expected results and output buffers first: everything below allocates nothing
    xs = [torch.remainder(torch.randint(0, 2 ** 62, (2, lv, n), device="cuda", generator=g), pr) for _ in range(2)]
    wants = [ctx.rescale(x) for x in xs]
    gots = [torch.full((2, lv - 1, n), -1, dtype=torch.int64, device="cuda") for _ in range(2)]
    empty = torch.zeros(1, dtype=torch.int64, device="cuda")
    big = torch.zeros(3, lv, n, dtype=torch.int64, device="cuda")
    before = _memory(L, ctx)
    for x, got in zip(xs, gots):  # two calls in a row, different inputs
        assert _noalloc(L, ctx, x, got, 2, lv) == 0, L.shm_last_error()
    # an empty batch does nothing and leaves no launch error for the next call
    assert _noalloc(L, ctx, empty, empty, 0, lv) == 0, L.shm_last_error()
    # beyond the fixed scratch: 2 polynomials x 24 limbs fit, 3 x 24 do not
    assert _noalloc(L, ctx, big, big, 3, lv) != 0
    assert b"fixed scratch" in L.shm_last_error()
    after = _memory(L, ctx)
    assert after == before, f"memory changed: {before} -> {after}"
    for got, want in zip(gots, wants):
        assert torch.equal(got, want)
    assert not torch.equal(gots[0], gots[1])
    # the call after the empty batch still succeeds (no pending launch error)
    again = torch.full_like(gots[0], -1)
    assert _noalloc(L, ctx, xs[0], again, 2, lv) == 0, L.shm_last_error()
    torch.cuda.synchronize()
    assert torch.equal(again, wants[0])
    ctx.close()
