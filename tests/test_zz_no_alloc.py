"""shm_rescale_noalloc: the rescale for callers that cannot allocate device
memory (a host whose own pool owns all device memory, a latency-critical path
that cannot take cudaMalloc's implicit synchronisation, an FFI caller without a
device allocator).  It must give exactly what shm_rescale gives (integer work:
bit for bit), on two calls in a row, and refuse sizes beyond its fixed scratch.

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


def test_rescale_noalloc_matches_rescale_on_two_calls():
    import torch

    from shmoai_b200._lib import lib
    from shmoai_b200.ckks import CKKSContext

    L = lib()
    L.shm_rescale_noalloc.restype = ctypes.c_int
    L.shm_rescale_noalloc.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_uint32] * 2 + [ctypes.c_void_p]
    L.shm_rescale_noalloc_max_words.restype = ctypes.c_size_t
    ctx = CKKSContext(16, bits=BITS, n_special=8)
    n, lv = ctx.n, ctx.nq
    assert L.shm_rescale_noalloc_max_words() * 8 == 32 << 20
    pr = torch.tensor(ctx.primes[:lv].astype(np.int64), device="cuda").view(1, lv, 1)
    g = torch.Generator(device="cuda").manual_seed(1)
    outs = []
    for _ in range(2):  # two calls in a row, different inputs
        x = torch.remainder(torch.randint(0, 2 ** 62, (2, lv, n), device="cuda", generator=g), pr)
        want = ctx.rescale(x)
        got = torch.full((2, lv - 1, n), -1, dtype=torch.int64, device="cuda")
        assert _noalloc(L, ctx, x, got, 2, lv) == 0, L.shm_last_error()
        torch.cuda.synchronize()
        assert torch.equal(got, want)
        outs.append(got)
    assert not torch.equal(outs[0], outs[1])
    # beyond the fixed scratch: 2 polynomials x 24 limbs fit, 3 x 24 do not
    big = torch.zeros(3, lv, n, dtype=torch.int64, device="cuda")
    assert _noalloc(L, ctx, big, big, 3, lv) != 0
    assert b"fixed scratch" in L.shm_last_error()
    ctx.close()
