"""shm_relinearize_rescale: relinearisation and rescale in one ModDown by S = q_{L-1} P with
an exact conversion (out = floor((P c + ks) / S)).

CPU: on the oracle's C ABI the result equals the reference's two-step sequence
(shm_relinearize then shm_rescale) bit for bit at every level, for random residues (the two
differ only where the sum lies within n_p + 1 of a multiple of q_{L-1} P, probability about
n_p / q_{L-1} per coefficient); without the overflow count the conversion would leave a
one-sided offset of up to n_p + 1 per coefficient, which summed over EvalMod's products
raised the worst slot error of a bootstrap fivefold.  Overlapping buffers and L = 1 are
refused.  GPU: the CUDA library against the oracle and against its own two-step sequence,
bit for bit, at every level of the small chain with several ciphertexts per call and at
three levels of the bootstrapping chain (N = 2^16).
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_CAPI = os.path.join(ROOT, "oracle", "_build", "libshmoai_oracle_capi.so")
P = ctypes.c_void_p
U32 = ctypes.c_uint32
SZ = ctypes.c_size_t


def _bind(lib):
    lib.shm_last_error.restype = ctypes.c_char_p
    lib.shm_context_create_from_primes.argtypes = [ctypes.POINTER(P), U32, ctypes.POINTER(ctypes.c_uint64), U32,
                                                   U32, ctypes.c_int]
    lib.shm_context_destroy.argtypes = [P]
    for name in ("shm_relinearize", "shm_relinearize_rescale"):
        getattr(lib, name).argtypes = [P, P, P, P, U32, U32, P, SZ, P]
    lib.shm_rescale.argtypes = [P, P, P, U32, U32, P, SZ, P]
    return lib


class Api:
    def __init__(self, lib, log_n, primes, n_special, device):
        self.lib, self.device, self.n = _bind(lib), device, 1 << log_n
        self.h = P()
        pr = np.ascontiguousarray(primes, dtype=np.uint64)
        rc = self.lib.shm_context_create_from_primes(ctypes.byref(self.h), log_n,
                                                     pr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                                     len(pr) - n_special, n_special, 0)
        assert rc == 0, self.lib.shm_last_error()
        self.keep = []

    def buf(self, a):
        if self.device:
            import torch
            t = torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()
        else:
            t = np.ascontiguousarray(a).copy()
        self.keep.append(t)
        return t

    def ptr(self, t):
        return t.data_ptr() if self.device else t.ctypes.data

    def host(self, t):
        if self.device:
            import torch
            torch.cuda.synchronize()
            return t.cpu().numpy().view(np.uint64).copy()
        return t.copy()

    def ok(self, rc):
        assert rc == 0, self.lib.shm_last_error()

    def fused(self, ct3, key, L):
        n_cts = ct3.shape[0]
        d3, dk = self.buf(ct3), self.buf(key)
        out = self.buf(np.zeros((n_cts, 2, L - 1, self.n), dtype=np.uint64))
        self.ok(self.lib.shm_relinearize_rescale(self.h, self.ptr(d3), self.ptr(dk), self.ptr(out), n_cts, L, None, 0,
                                                 None))
        return self.host(out)

    def two_step(self, ct3, key, L):
        n_cts = ct3.shape[0]
        d3, dk = self.buf(ct3), self.buf(key)
        r = self.buf(np.zeros((n_cts, 2, L, self.n), dtype=np.uint64))
        self.ok(self.lib.shm_relinearize(self.h, self.ptr(d3), self.ptr(dk), self.ptr(r), n_cts, L, None, 0, None))
        out = self.buf(np.zeros((n_cts, 2, L - 1, self.n), dtype=np.uint64))
        self.ok(self.lib.shm_rescale(self.h, self.ptr(r), self.ptr(out), n_cts * 2, L, None, 0, None))
        return self.host(out)

    def close(self):
        self.lib.shm_context_destroy(self.h)


# the N = 2^12 chain of six primes, and the bootstrapping chain's primes at N = 2^12
SETS = {"tiny": O.PARAM_SETS["tiny"], "boot4k": (12, [51] + [46] * 20 + [51] * 14 + [51] * 5, 5)}


def _rand(rng, shape, primes):
    out = np.empty(shape, dtype=np.uint64)
    for i, q in enumerate(primes):
        out[..., i, :] = rng.integers(0, q, size=shape[:-2] + (shape[-1],), dtype=np.uint64)
    return out


def _case(rng, primes, nq, np_, L, n_cts, n):
    dnum = nq // np_
    ct3 = _rand(rng, (n_cts, 3, L, n), primes[:L])
    key = _rand(rng, (dnum, 2, nq + np_, n), primes)
    return ct3, key


@pytest.mark.parametrize("pset,L", [("tiny", 2), ("tiny", 3), ("tiny", 5), ("tiny", 6), ("boot4k", 2), ("boot4k", 9),
                                     ("boot4k", 20)])
def test_oracle_fused_equals_the_two_step_sequence(pset, L):
    log_n, bits, np_ = SETS[pset]
    primes = [int(p) for p in O.gen_primes(log_n, bits)]
    nq = len(primes) - np_
    api = Api(ctypes.CDLL(ORACLE_CAPI), log_n, primes, np_, device=False)
    rng = np.random.default_rng(100 + L)
    ct3, key = _case(rng, primes, nq, np_, L, 2, api.n)
    assert np.array_equal(api.fused(ct3, key, L), api.two_step(ct3, key, L))
    api.close()


def test_oracle_refuses_overlap_and_level_one():
    log_n, bits, np_ = O.PARAM_SETS["tiny"]
    primes = [int(p) for p in O.gen_primes(log_n, bits)]
    api = Api(ctypes.CDLL(ORACLE_CAPI), log_n, primes, np_, device=False)
    rng = np.random.default_rng(3)
    ct3, key = _case(rng, primes, len(primes) - np_, np_, 3, 1, api.n)
    d3, dk = api.buf(ct3), api.buf(key)
    assert api.lib.shm_relinearize_rescale(api.h, api.ptr(d3), api.ptr(dk), api.ptr(d3), 1, 3, None, 0, None) != 0
    assert b"overlap" in api.lib.shm_last_error()
    out = api.buf(np.zeros((1, 2, 1, api.n), dtype=np.uint64))
    assert api.lib.shm_relinearize_rescale(api.h, api.ptr(d3), api.ptr(dk), api.ptr(out), 1, 1, None, 0, None) != 0
    api.close()


@pytest.mark.gpu
@pytest.mark.parametrize("pset,levels,n_cts", [("tiny", [2, 3, 4, 5, 6], 3), ("boot", [2, 13, 35], 1)])
def test_cuda_relinearize_rescale_matches_oracle(pset, levels, n_cts):
    import shmoai_b200

    log_n, bits, np_ = O.PARAM_SETS[pset]
    primes = [int(p) for p in O.gen_primes(log_n, bits)]
    nq = len(primes) - np_
    cu = Api(shmoai_b200.lib(), log_n, primes, np_, device=True)
    orc = Api(ctypes.CDLL(ORACLE_CAPI), log_n, primes, np_, device=False)
    for L in levels:
        rng = np.random.default_rng(7 * L)
        ct3, key = _case(rng, primes, nq, np_, L, n_cts, cu.n)
        got = cu.fused(ct3, key, L)
        assert np.array_equal(got, orc.fused(ct3, key, L)), L
        assert np.array_equal(got, cu.two_step(ct3, key, L)), L
        cu.keep.clear()
    cu.close()
    orc.close()
