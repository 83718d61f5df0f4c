"""Attention's ciphertext-ciphertext products (src/include/source/matrix_mul/Ct_ct_matrix_mul.cuh):
the column packing (shm_host_ct_ct_matmul; ct_ct_matrix_mul_colpacking, :10-120),
out_i = sum_j X_j * rot(W_j, i * num_batch), and the diagonal packing (shm_host_ct_ct_matmul_diag;
ct_ct_matrix_mul_diagpacking, :182-), a baby-step giant-step product over X's diagonals; one
relinearisation and rescale per output (per giant step for the diagonal packing).

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


def _diag_want(X, W, nb):
    """ct_ct_matrix_mul_diagpacking's arithmetic on slot vectors (Ct_ct_matrix_mul.cuh:182-)."""
    col, n = len(X), X.shape[1]
    g = int(np.ceil(np.sqrt(col)))
    b = -(-col // g)
    rot = lambda v, k: np.roll(v, -(k % n))
    rx = [rot(X[i], (col - (i // g) * g) * nb) if i >= g else X[i] for i in range(col)]
    out = []
    for w in W:
        total = 0
        for j in range(b):
            acc = sum(rot(w, k * nb) * rx[j * g + k] for k in range(g) if j * g + k < col)
            total = total + rot(acc, j * g * nb)
        out.append(total)
    return np.stack(out)


def _diag_steps(col, nb, n):
    g = int(np.ceil(np.sqrt(col)))
    b = -(-col // g)
    st = {(col - i * g) * nb % n for i in range(1, b)} | {j * nb % n for j in range(1, g)}
    st |= {j * g * nb % n for j in range(1, b)}
    return sorted(s for s in st if s)


@pytest.mark.parametrize("col,cw", [(4, 2), (7, 3), (9, 1)])
def test_ct_ct_matmul_diag_matches_the_slot_arithmetic(col, cw):
    nb = 16
    h = Host(12, O.gen_primes(12, BITS), 5, hamming_weight=64, seed=13, lib=ORACLE_HOST)
    h.gen_relin_key()
    h.gen_galois_keys([h.galois_elt(s) for s in _diag_steps(col, nb, h.n // 2)])
    rng = np.random.default_rng(col * 10 + cw)
    X, W = rng.uniform(-1, 1, (col, h.n // 2)), rng.uniform(-1, 1, (cw, h.n // 2))
    out = h.ct_ct_matmul_diag(h.encrypt(X, DELTA, 6), h.encrypt(W, DELTA, 6), nb)
    assert (out.count, out.level) == (cw, 5)
    assert np.abs(h.decrypt(out).real - _diag_want(X, W, nb)).max() < 1e-7


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
    for h in (g, c):
        h.gen_galois_keys([h.galois_elt(st) for st in _diag_steps(7, 16, h.n // 2)])
    Xd = rng.uniform(-1, 1, (7, g.n // 2))
    a = g.ct_ct_matmul_diag(g.encrypt(Xd, DELTA, 6), g.encrypt(W, DELTA, 6), 16)
    b = c.ct_ct_matmul_diag(c.encrypt(Xd, DELTA, 6), c.encrypt(W, DELTA, 6), 16)
    assert np.array_equal(a.to_host(), b.to_host())
