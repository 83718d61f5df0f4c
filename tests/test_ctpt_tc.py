"""Tensor-core ct-pt matmul (small-modulus residue system on tcgen05 kind::i8)
against the CUDA-core contraction and the CPU oracle, at ragged shapes (K not a
multiple of 64, more than one 256-output tile, large and negative weights)."""
import numpy as np
import pytest

from golden.golden import GoldenSet
from oracle import oracle as O

pytestmark = pytest.mark.gpu


# K up to 768 runs the persistent kernel (X tile resident in shared memory); 800 inputs (K padded
# to 832) the tile-per-CTA kernel
@pytest.mark.parametrize("n_in,n_out,wbits", [(8, 4, 36), (200, 300, 39), (64, 256, 20), (130, 17, 39),
                                              (768, 130, 30), (800, 40, 30)])
def test_tc_matches_cuda_core_and_oracle(n_in, n_out, wbits):
    import ctypes

    import torch

    from shmoai_b200._lib import check, lib
    from shmoai_b200.ckks import CKKSContext, to_device, to_host

    g = GoldenSet("tiny")
    ctx = CKKSContext(g.log_n, primes=g.primes, n_special=g.np)
    L = g.L
    rng = np.random.default_rng(n_in * 1000 + n_out)
    X = np.stack([g.ct(3000 + i, L) for i in range(n_in)])
    W = rng.integers(-(1 << wbits), 1 << wbits, size=(n_in, n_out), dtype=np.int64)
    W[0, 0] = (1 << wbits) - 1
    W[-1, -1] = -(1 << wbits)
    Xd, Wd = to_device(X), torch.from_numpy(W).cuda()
    Y = to_host(ctx.ctpt_matmul(Xd, Wd))
    Yc = torch.empty(n_out, 2, L, g.n, dtype=torch.int64, device="cuda")
    check(lib().shm_ctpt_matmul_cuda_core(ctx._h, ctypes.c_void_p(Xd.data_ptr()), ctypes.c_void_p(Wd.data_ptr()),
                                          ctypes.c_void_p(Yc.data_ptr()), n_in, n_out, L,
                                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    assert np.array_equal(Y, to_host(Yc))
    o = O.Oracle(g.log_n, g.primes, g.nq, g.np)
    cols = [0, n_out - 1]
    ref = o.ctpt_matmul(X, np.ascontiguousarray(W[:, cols]))
    for k, c in enumerate(cols):
        assert np.array_equal(Y[c], ref[k])
    ctx.close()


@pytest.mark.parametrize("L", [2, 3])
def test_tc_over_several_column_chunks(L):
    """N = 2^16: 2 L N columns are two or three chunks of 131,072 columns, each its own pass
    of residues, GEMM and CRT (the weight planes and the CRT table shared)."""
    import ctypes

    import torch

    from shmoai_b200._lib import check, lib
    from shmoai_b200.ckks import CKKSContext, to_device, to_host

    log_n, bits, np_ = O.PARAM_SETS["boot"]
    primes = [int(p) for p in O.gen_primes(log_n, bits)]
    ctx = CKKSContext(log_n, primes=primes, n_special=np_)
    n, n_in, n_out = 1 << log_n, 24, 9
    rng = np.random.default_rng(40 + L)
    X = np.empty((n_in, 2, L, n), dtype=np.uint64)
    for l in range(L):
        X[:, :, l] = rng.integers(0, primes[l], size=(n_in, 2, n), dtype=np.uint64)
    W = rng.integers(-(1 << 30), 1 << 30, size=(n_in, n_out), dtype=np.int64)
    Xd, Wd = to_device(X), torch.from_numpy(W).cuda()
    Y = to_host(ctx.ctpt_matmul(Xd, Wd))
    Yc = torch.empty(n_out, 2, L, n, dtype=torch.int64, device="cuda")
    check(lib().shm_ctpt_matmul_cuda_core(ctx._h, ctypes.c_void_p(Xd.data_ptr()), ctypes.c_void_p(Wd.data_ptr()),
                                          ctypes.c_void_p(Yc.data_ptr()), n_in, n_out, L,
                                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    assert np.array_equal(Y, to_host(Yc))
    o = O.Oracle(log_n, primes, len(primes) - np_, np_)
    ref = o.ctpt_matmul(X, np.ascontiguousarray(W[:, [0, n_out - 1]]))
    assert np.array_equal(Y[0], ref[0]) and np.array_equal(Y[n_out - 1], ref[1])
    ctx.close()
