"""The MOAI packing of a batch of inputs (src/include/source/matrix_mul/Batch_encode_encrypt.cuh):
batch_input's column-interleaved layout under public-key encryption and bias_vec's slot mask,
against numpy restatements of the reference's index arithmetic (:12-56)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from shmoai_b200.host import Host, HostError, bias_vec

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_HOST = os.path.join(ROOT, "oracle", "_build", "libshmoai_host_oracle.so")


def _reference_packing(X):
    """vec[num_X * k + j] = X[j][k][i] for column i (Batch_encode_encrypt.cuh:29-35)."""
    nx, nr, nc = X.shape
    out = np.zeros((nc, nx * nr))
    for i in range(nc):
        for j in range(nx):
            for k in range(nr):
                out[i, nx * k + j] = X[j, k, i]
    return out


def _reference_bias_vec(lengths, nx, nr):
    out = np.zeros(nx * nr, dtype=np.int32)
    for i in range(nx):
        for j in range(lengths[i]):
            out[j * nx + i] = 1
    return out


def _packing_case(lib):
    log_n, bits, n_sp = O.PARAM_SETS["tiny"]
    h = Host(log_n, bits=bits, n_special=n_sp, hamming_weight=64, seed=5, lib=lib)
    h.gen_public_key(3)
    rng = np.random.default_rng(9)
    nx, nr, nc = 8, 128, 6  # 1,024 of 2,048 slots used
    X = np.clip(rng.normal(size=(nx, nr, nc)), -4, 4)
    ct = h.batch_input(X, 2.0 ** 40, h.nq)
    assert (ct.count, ct.level) == (nc, h.nq)
    got = h.decrypt(ct)
    want = np.zeros((nc, h.n // 2))
    want[:, : nx * nr] = _reference_packing(X)
    assert np.abs(got - want).max() < 1e-6
    return ct.to_host()


def test_batch_input_matches_reference_layout():
    _packing_case(ORACLE_HOST)


def test_bias_vec_matches_reference():
    lengths = [128, 3, 0, 77, 128, 1, 64, 100]
    got = bias_vec(lengths, 8, 128, ORACLE_HOST)
    assert np.array_equal(got, _reference_bias_vec(lengths, 8, 128))
    with pytest.raises(HostError):
        bias_vec([129] * 8, 8, 128, ORACLE_HOST)


@pytest.mark.gpu
def test_batch_input_cuda_matches_oracle_build():
    assert np.array_equal(_packing_case(None), _packing_case(ORACLE_HOST))


def _masked_case(lib):
    """The masked projection (ct_pt_matrix_mul_wo_pre_w_mask, Ct_pt_matrix_mul.cuh:846-986) on the packing:
    Y[o] = bias_vec * sum_i X[i] W[i][o], slot-wise."""
    log_n, bits, n_sp = O.PARAM_SETS["tiny"]
    h = Host(log_n, bits=bits, n_special=n_sp, hamming_weight=64, seed=6, lib=lib)
    h.gen_public_key(4)
    rng = np.random.default_rng(10)
    nx, nr, n_in, n_out = 16, 128, 12, 5
    X = np.clip(rng.normal(size=(nx, nr, n_in)), -4, 4)
    ct = h.batch_input(X, 2.0 ** 50, h.nq)  # x 2^40 weights / a 50-bit prime: products at 2^40
    w_scale = 2.0 ** 40
    W = np.round(rng.normal(0, 0.02, (n_in, n_out)) * w_scale).astype(np.int64)
    lengths = rng.integers(1, nr + 1, nx)
    mask = bias_vec(lengths, nx, nr, lib).astype(np.float64)
    Y = h.ctpt_matmul_masked(ct, W, w_scale, mask)
    assert (Y.count, Y.level) == (n_out, h.nq - 2)
    xs = _reference_packing(X)  # [n_in][slots]
    want = mask[None, :] * ((W.astype(np.float64) / w_scale).T @ xs)
    got = h.decrypt(Y)[:, : nx * nr]
    assert np.abs(got - want).max() < 1e-6
    return Y.to_host()


def test_masked_projection_on_oracle():
    _masked_case(ORACLE_HOST)


@pytest.mark.gpu
def test_masked_projection_cuda_matches_oracle_build():
    assert np.array_equal(_masked_case(None), _masked_case(ORACLE_HOST))
