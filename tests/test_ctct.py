"""Attention's ciphertext-ciphertext product in the column packing (shm_host_ct_ct_matmul;
ct_ct_matrix_mul_colpacking, src/include/source/matrix_mul/Ct_ct_matrix_mul.cuh:10-120):
out_i = sum_j X_j * rot(W_j, i * num_batch), one relinearisation and rescale per output row.

CPU: the host library on the oracle's C ABI at N = 2^12; decryptions equal numpy's product of
the slot vectors with W's rows rotated (np.roll by -i * num_batch), for ragged column counts;
one level is used; mismatched batches and missing Galois keys are refused.  GPU: the CUDA
build equals the oracle build bit for bit.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from shmoai_b200.host import Host, HostError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_HOST = os.path.join(ROOT, "oracle", "_build", "libshmoai_host_oracle.so")
BITS = [51] + [46] * 8 + [51] + [51] * 5  # N = 2^12, nq = 10, np = 5
DELTA = 2.0 ** 46


def _host(lib=ORACLE_HOST, seed=11, rows=5, nb=16):
    h = Host(12, O.gen_primes(12, BITS), 5, hamming_weight=64, seed=seed, lib=lib)
    h.gen_relin_key()
    h.gen_galois_keys([h.galois_elt(i * nb) for i in range(1, rows)])
    return h


def _want(X, W, rows, nb):
    return np.stack([sum(X[j] * np.roll(W[j], -i * nb) for j in range(len(X))) for i in range(rows)])


@pytest.mark.parametrize("col", [1, 3, 4])
def test_ct_ct_matmul_matches_the_slot_product(col):
    rows, nb = 5, 16
    h = _host(rows=rows, nb=nb)
    rng = np.random.default_rng(col)
    X, W = rng.uniform(-1, 1, (col, h.n // 2)), rng.uniform(-1, 1, (col, h.n // 2))
    out = h.ct_ct_matmul(h.encrypt(X, DELTA, 6), h.encrypt(W, DELTA, 6), rows, nb)
    assert (out.count, out.level) == (rows, 5)
    assert np.abs(h.decrypt(out).real - _want(X, W, rows, nb)).max() < 1e-7


def test_ct_ct_matmul_refuses_bad_inputs():
    h = _host(rows=3, nb=16)
    rng = np.random.default_rng(9)
    X = h.encrypt(rng.uniform(-1, 1, (2, 64)), DELTA, 6)
    with pytest.raises(HostError, match="same number of columns"):
        h.ct_ct_matmul(X, h.encrypt(rng.uniform(-1, 1, (3, 64)), DELTA, 6), 3, 16)
    with pytest.raises(HostError, match="Galois key"):
        h.ct_ct_matmul(X, X, 5, 16)  # steps 48 and 64 have no keys


@pytest.mark.gpu
def test_cuda_ct_ct_matmul_matches_oracle_build():
    import shmoai_b200.host as H

    g, c = _host(lib=H.PRODUCT_LIB, seed=21), _host(seed=21)
    rng = np.random.default_rng(5)
    X, W = rng.uniform(-1, 1, (3, g.n // 2)), rng.uniform(-1, 1, (3, g.n // 2))
    a = g.ct_ct_matmul(g.encrypt(X, DELTA, 6), g.encrypt(W, DELTA, 6), 5, 16)
    b = c.ct_ct_matmul(c.encrypt(X, DELTA, 6), c.encrypt(W, DELTA, 6), 5, 16)
    assert np.array_equal(a.to_host(), b.to_host())
