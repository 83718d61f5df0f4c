"""Fused element-wise entry points of the EvalMod path: shm_linear_combination (a
polynomial leaf's weighted sum of Chebyshev basis ciphertexts plus its constant, in one
pass) and shm_add_sizes (an unrelinearised product plus an ordinary ciphertext); and of the
attention's ct-ct products: shm_multiply_accumulate (a sum of size-3 tensor products in one
pass, paired or with one broadcast ciphertext).

CPU: the oracle's C ABI against exact Python integer arithmetic.  GPU: the CUDA library
against the oracle's C ABI on the same inputs, bit for bit.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_CAPI = os.path.join(ROOT, "oracle", "_build", "libshmoai_oracle_capi.so")
BITS = [51, 46, 46, 51, 51]  # N = 2^12, nq = 4, np = 1
LOG_N = 12
P = ctypes.c_void_p
U64P = ctypes.POINTER(ctypes.c_uint64)


def _bind(lib):
    lib.shm_last_error.restype = ctypes.c_char_p
    lib.shm_context_create_from_primes.argtypes = [ctypes.POINTER(P), ctypes.c_uint32, U64P, ctypes.c_uint32,
                                                   ctypes.c_uint32, ctypes.c_int]
    lib.shm_context_destroy.argtypes = [P]
    lib.shm_linear_combination.argtypes = [P, ctypes.POINTER(P), ctypes.POINTER(ctypes.c_uint32), U64P,
                                           ctypes.c_uint32, U64P, P, ctypes.c_uint32, ctypes.c_uint32, P]
    lib.shm_add_sizes.argtypes = [P, P, ctypes.c_uint32, P, ctypes.c_uint32, P, ctypes.c_uint32, ctypes.c_uint32, P]
    lib.shm_multiply_accumulate.argtypes = [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.c_uint32, ctypes.c_int, P,
                                            ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, P]
    return lib


def _ctx(lib, primes, n_special=1):
    h = P()
    pr = np.ascontiguousarray(primes, dtype=np.uint64)
    assert lib.shm_context_create_from_primes(ctypes.byref(h), LOG_N, pr.ctypes.data_as(U64P), len(pr) - n_special,
                                              n_special, 0) == 0
    return h


def _case(seed, count=3, k=5, L=3):
    """Terms at 4, 3 and 4 primes (read at their first L), weights, constant residues."""
    primes = O.gen_primes(LOG_N, BITS)
    rng = np.random.default_rng(seed)
    n = 1 << LOG_N
    levels = [4, 3, 4, 4, 3][:k]
    X = [np.stack([rng.integers(0, primes[l], (count, 2, n), dtype=np.uint64) for l in range(lv)], axis=2)
         for lv in levels]
    w = np.array([[rng.integers(0, primes[l]) for l in range(L)] for _ in range(k)], dtype=np.uint64)
    w0 = np.array([rng.integers(0, primes[l]) for l in range(L)], dtype=np.uint64)
    return primes, [np.ascontiguousarray(x) for x in X], levels, w, w0


def _expected(primes, X, w, w0, L):
    count, n = X[0].shape[0], X[0].shape[-1]
    out = np.zeros((count, 2, L, n), dtype=np.uint64)
    for l in range(L):
        q = int(primes[l])
        acc = np.zeros((count, 2, n), dtype=object)
        for t in range(len(X)):
            acc = acc + X[t][:, :, l, :].astype(object) * int(w[t, l])
        acc[:, 0, :] += int(w0[l])
        out[:, :, l, :] = (acc % q).astype(np.uint64)
    return out


def _oracle_lin(primes, X, levels, w, w0, L):
    lib = _bind(ctypes.CDLL(ORACLE_CAPI))
    h = _ctx(lib, primes)
    count, n = X[0].shape[0], X[0].shape[-1]
    out = np.zeros((count, 2, L, n), dtype=np.uint64)
    ptrs = (P * len(X))(*[x.ctypes.data for x in X])
    lv = (ctypes.c_uint32 * len(X))(*levels)
    wf = np.ascontiguousarray(w)
    rc = lib.shm_linear_combination(h, ptrs, lv, wf.ctypes.data_as(U64P), len(X), w0.ctypes.data_as(U64P),
                                    out.ctypes.data, count, L, None)
    lib.shm_context_destroy(h)
    assert rc == 0, lib.shm_last_error()
    return out


def _oracle_add_sizes(primes, a, b, L):
    lib = _bind(ctypes.CDLL(ORACLE_CAPI))
    h = _ctx(lib, primes)
    out = np.zeros_like(a)
    rc = lib.shm_add_sizes(h, a.ctypes.data, a.shape[1], b.ctypes.data, b.shape[1], out.ctypes.data, a.shape[0], L,
                           None)
    lib.shm_context_destroy(h)
    assert rc == 0, lib.shm_last_error()
    return out


def test_oracle_linear_combination_is_the_exact_sum():
    primes, X, levels, w, w0 = _case(1)
    assert np.array_equal(_oracle_lin(primes, X, levels, w, w0, 3), _expected(primes, X, w, w0, 3))


def test_oracle_add_sizes():
    primes = O.gen_primes(LOG_N, BITS)
    rng = np.random.default_rng(2)
    L, n = 3, 1 << LOG_N
    q = np.array(primes[:L], dtype=np.uint64).reshape(1, 1, L, 1)
    a = (rng.integers(0, 2 ** 62, (2, 3, L, n), dtype=np.uint64) % q).astype(np.uint64)
    b = (rng.integers(0, 2 ** 62, (2, 2, L, n), dtype=np.uint64) % q).astype(np.uint64)
    want = a.copy()
    want[:, :2] = ((a[:, :2].astype(object) + b.astype(object)) % q.astype(object)).astype(np.uint64)
    assert np.array_equal(_oracle_add_sizes(primes, a, b, L), want)


@pytest.mark.gpu
def test_cuda_fused_ops_match_oracle():
    import torch

    import shmoai_b200

    lib = _bind(shmoai_b200.lib())
    for seed in (3, 4):
        primes, X, levels, w, w0 = _case(seed)
        h = _ctx(lib, primes)
        dX = [torch.from_numpy(x.view(np.int64)).cuda() for x in X]
        out = torch.empty((X[0].shape[0], 2, 3, 1 << LOG_N), dtype=torch.int64, device="cuda")
        ptrs = (P * len(dX))(*[t.data_ptr() for t in dX])
        lv = (ctypes.c_uint32 * len(dX))(*levels)
        wf = np.ascontiguousarray(w)
        rc = lib.shm_linear_combination(h, ptrs, lv, wf.ctypes.data_as(U64P), len(dX), w0.ctypes.data_as(U64P),
                                        out.data_ptr(), X[0].shape[0], 3, None)
        assert rc == 0, lib.shm_last_error()
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint64), _oracle_lin(primes, X, levels, w, w0, 3))

        a, b = X[0][:, :, :3].copy(), X[2][:, :, :3].copy()
        a3 = np.ascontiguousarray(np.concatenate([a, a[:, :1]], axis=1))  # [count][3][L][N]
        da, db = torch.from_numpy(a3.view(np.int64)).cuda(), torch.from_numpy(np.ascontiguousarray(b).view(np.int64)).cuda()
        do = torch.empty_like(da)
        rc = lib.shm_add_sizes(h, da.data_ptr(), 3, db.data_ptr(), 2, do.data_ptr(), a3.shape[0], 3, None)
        assert rc == 0, lib.shm_last_error()
        torch.cuda.synchronize()
        assert np.array_equal(do.cpu().numpy().view(np.uint64), _oracle_add_sizes(primes, a3, np.ascontiguousarray(b), 3))
        lib.shm_context_destroy(h)


# ---- shm_multiply_accumulate: out[c] = sum_t A_t[c] x B_t[c or 0]

# a chain with 60-bit primes too: 2k products of 120 bits overflow the Barrett bound past k = 4,
# so the entry point splits the terms and accumulates
BITS60 = [60, 50, 60, 60]


def _mac_case(seed, bits, count, k, L, bcast):
    primes = O.gen_primes(LOG_N, bits)
    rng = np.random.default_rng(seed)
    n = 1 << LOG_N
    q = np.array(primes[:L], dtype=np.uint64).reshape(1, 1, L, 1)
    A = [np.ascontiguousarray(rng.integers(0, 2 ** 63, (count, 2, L, n), dtype=np.uint64) % q) for _ in range(k)]
    B = [np.ascontiguousarray(rng.integers(0, 2 ** 63, (1 if bcast else count, 2, L, n), dtype=np.uint64) % q)
         for _ in range(k)]
    return primes, A, B


def _mac_expected(primes, A, B, L, bcast):
    count, n = A[0].shape[0], A[0].shape[-1]
    q = np.array([int(x) for x in primes[:L]], dtype=object).reshape(1, L, 1)
    s = [np.zeros((count, L, n), dtype=object) for _ in range(3)]
    for a, b in zip(A, B):
        a0, a1 = a[:, 0].astype(object), a[:, 1].astype(object)
        b0, b1 = b[:, 0].astype(object), b[:, 1].astype(object)
        s[0] = s[0] + a0 * b0
        s[1] = s[1] + a0 * b1 + a1 * b0
        s[2] = s[2] + a1 * b1
    return np.stack([(x % q).astype(np.uint64) for x in s], axis=1)


def _mac_call(lib, h, A, B, count, L, bcast, arrays):
    out = arrays.empty(count, L)
    pa = (P * len(A))(*[arrays.ptr(a) for a in A])
    pb = (P * len(B))(*[arrays.ptr(b) for b in B])
    rc = lib.shm_multiply_accumulate(h, pa, pb, len(A), 1 if bcast else 0, arrays.ptr(out), count, L, 0, None)
    assert rc == 0, lib.shm_last_error()
    return arrays.host(out)


class _HostArrays:
    @staticmethod
    def empty(count, L):
        return np.zeros((count, 3, L, 1 << LOG_N), dtype=np.uint64)

    @staticmethod
    def ptr(a):
        return a.ctypes.data

    @staticmethod
    def host(a):
        return a


def _oracle_mac(primes, A, B, L, bcast, n_special):
    lib = _bind(ctypes.CDLL(ORACLE_CAPI))
    h = _ctx(lib, primes, n_special)
    try:
        return _mac_call(lib, h, A, B, A[0].shape[0], L, bcast, _HostArrays)
    finally:
        lib.shm_context_destroy(h)


@pytest.mark.parametrize("bits,k,bcast", [(BITS, 5, False), (BITS, 3, True), (BITS60, 6, False)])
def test_oracle_multiply_accumulate_is_the_exact_sum(bits, k, bcast):
    L = 3
    primes, A, B = _mac_case(7, bits, 2, k, L, bcast)
    assert np.array_equal(_oracle_mac(primes, A, B, L, bcast, 1), _mac_expected(primes, A, B, L, bcast))


@pytest.mark.gpu
def test_cuda_multiply_accumulate_matches_oracle():
    import torch

    import shmoai_b200

    class Dev:
        keep = []

        @staticmethod
        def empty(count, L):
            return torch.empty((count, 3, L, 1 << LOG_N), dtype=torch.int64, device="cuda")

        @classmethod
        def ptr(cls, a):
            if isinstance(a, np.ndarray):
                a = torch.from_numpy(a.view(np.int64)).cuda()
                cls.keep.append(a)
            return a.data_ptr()

        @staticmethod
        def host(a):
            torch.cuda.synchronize()
            return a.cpu().numpy().view(np.uint64)

    lib = _bind(shmoai_b200.lib())
    # 40 paired terms (more than one launch's 32), a broadcast term list, and the 60-bit chain
    for seed, bits, count, k, bcast in ((8, BITS, 3, 40, False), (9, BITS, 4, 12, True), (10, BITS60, 2, 9, False)):
        L = 3
        primes, A, B = _mac_case(seed, bits, count, k, L, bcast)
        h = _ctx(lib, primes)
        got = _mac_call(lib, h, A, B, count, L, bcast, Dev)
        lib.shm_context_destroy(h)
        Dev.keep.clear()
        assert np.array_equal(got, _oracle_mac(primes, A, B, L, bcast, 1)), (seed, k, bcast)
