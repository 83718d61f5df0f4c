"""Polynomial operators of the BERT layer on ciphertext batches (shm_host_chebyshev,
shm_host_gelu, shm_host_exp, shm_host_inverse, shm_host_inv_sqrt, shm_host_layernorm,
shm_host_softmax; the
reference's non_linear_func/: gelu_cheb at gelu_other.cuh:258-300, exp and inverse at
softmax.cuh:23-118, invert_sqrt and layernorm in layernorm.cuh).

CPU: the host library on the oracle's C ABI at N = 2^12.  A Chebyshev series evaluated on
ciphertexts decrypts to numpy's evaluation of the same series (CKKS noise only); GELU
decrypts to the reference's degree-24 series and, through it, to GELU within the series'
fit error on [-19.5, 12.5] (0.037 in the reference's own comment; checked here against
x Phi(x)); bad inputs are refused.  GPU: the CUDA build gives the oracle build's results
bit for bit, and GELU at N = 2^16 on the bootstrapping chain has the same accuracy.
"""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from shmoai_b200.host import Host, HostError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_HOST = os.path.join(ROOT, "oracle", "_build", "libshmoai_host_oracle.so")
SMALL_BITS = [51] + [46] * 8 + [51] * 11 + [51] * 5  # N = 2^12, nq = 20, np = 5
REF_BITS = [51] + [46] * 20 + [51] * 14 + [51] * 5
DELTA = 2.0 ** 46
# gelu_cheb's series in u = (x + 3.5) / 16 (gelu_other.cuh:284-296), as the operator uses it
GELU_D = [3.4550752799e+00, 5.7852067632e+00, 3.1727714170e+00, 7.0234932500e-01, -4.6200569546e-01,
          -3.7817535966e-01, 8.4136420694e-02, 2.2427456987e-01, 2.9451916291e-02, -1.2928072669e-01,
          -6.6659430283e-02, 6.4349502364e-02, 7.1733295078e-02, -1.9882581810e-02, -6.1145844240e-02,
          -8.4827295421e-03, 4.3597254356e-02, 2.3373027950e-02, -2.4790187963e-02, -2.7940100474e-02,
          8.8404026343e-03, 2.3776567058e-02, 8.8171887083e-03, -4.6290425955e-02, -9.7997267900e-03]


def _gelu(x):
    return 0.5 * x * (1.0 + np.vectorize(math.erf)(x / math.sqrt(2.0)))


def _host(lib=ORACLE_HOST, seed=11, log_n=12, bits=SMALL_BITS, hw=64):
    h = Host(log_n, O.gen_primes(log_n, bits), 5, hamming_weight=hw, seed=seed, lib=lib)
    h.gen_relin_key()
    return h


@pytest.fixture(scope="module")
def small():
    return _host()


@pytest.mark.parametrize("deg,L", [(5, 6), (12, 7), (24, 9)])
def test_chebyshev_series_matches_numpy(small, deg, L):
    h = small
    rng = np.random.default_rng(deg)
    lo, hi = -3.0, 5.0
    c = rng.uniform(-1, 1, deg + 1) / (1 + np.arange(deg + 1))
    x = rng.uniform(lo, hi, (2, h.n // 2))
    out = h.chebyshev(h.encrypt(x, DELTA, L), c, lo, hi)
    want = np.polynomial.chebyshev.chebval((2 * x - hi - lo) / (hi - lo), c)
    assert out.scale == DELTA and out.level < L
    assert np.abs(h.decrypt(out).real - want).max() < 1e-5


def test_gelu_is_the_reference_series(small):
    h = small
    rng = np.random.default_rng(3)
    x = rng.uniform(-19.5, 12.5, (2, h.n // 2))
    x[0, :4] = [-19.5, 12.5, 0.0, -3.5]
    out = h.gelu(h.encrypt(x, DELTA, 9))
    y = h.decrypt(out).real
    series = np.polynomial.chebyshev.chebval((x + 3.5) / 16.0, GELU_D)
    assert out.level == 9 - 6 and out.scale == DELTA  # one level fewer than gelu_cheb's 7
    assert np.abs(y - series).max() < 1e-5
    assert np.abs(y - _gelu(x)).max() < 0.04


def test_exp_and_inverse_are_the_reference_formulas(small):
    """exp as (1 + x/128)^128 and 1/x as prod (1 + (1 - x)^(2^i)) (softmax.cuh:23-118):
    decryptions equal numpy's evaluation of the same formulas; levels 8 and iter + 1."""
    h = small
    rng = np.random.default_rng(8)
    x = rng.uniform(-8.0, 1.0, (2, h.n // 2))
    out = h.exp(h.encrypt(x, DELTA, 10))
    assert out.level == 2
    assert np.abs(h.decrypt(out).real - (1 + x / 128) ** 128).max() < 1e-6
    x = rng.uniform(0.05, 1.95, (2, h.n // 2))
    for it in (3, 7):
        out = h.inverse(h.encrypt(x, DELTA, 9), it)
        y, r = 1 - x, 2 - x
        for _ in range(it):
            y = y * y
            r = r * (1 + y)
        assert out.level == 9 - it - 1
        assert np.abs(h.decrypt(out).real - r).max() < 1e-6
    assert h.exp(h.encrypt(x - 1.0, DELTA, 9)).level == 1
    with pytest.raises(HostError, match="levels"):
        h.exp(h.encrypt(x, DELTA, 8))
    with pytest.raises(HostError, match="levels"):
        h.inverse(h.encrypt(x, DELTA, 5), 4)


def _inv_sqrt_reference(x, d_newt=4, d_gold=2):
    """invert_sqrt's arithmetic in numpy (layernorm.cuh:708-897)."""
    r = -1.29054537e-4 * x + 1.29054537e-1
    for _ in range(d_newt):
        r = r * (1.5 - 0.5 * x * r * r)
    g, h = x * r, 0.5 * r
    for _ in range(d_gold):
        s = 0.5 - g * h
        g, h = g + g * s, h + h * s
    return 2 * h


def test_inv_sqrt_is_the_reference_iteration():
    """LayerNorm's inverse square root: a linear guess, 4 Newton and 2 Goldschmidt steps,
    2 (d_newt + d_gold) + 3 levels; decryptions equal numpy's run of the same iteration."""
    h = _host(bits=[51] + [46] * 19 + [51] + [51] * 5)
    rng = np.random.default_rng(9)
    x = rng.uniform(1.0, 800.0, (2, h.n // 2))
    out = h.inv_sqrt(h.encrypt(x, DELTA, 21))
    assert out.level == 21 - 15 and out.scale == DELTA
    assert np.abs(h.decrypt(out).real - _inv_sqrt_reference(x)).max() < 1e-7
    out = h.inv_sqrt(h.encrypt(x, DELTA, 16), 2, 1)
    assert out.level == 16 - 9
    assert np.abs(h.decrypt(out).real - _inv_sqrt_reference(x, 2, 1)).max() < 1e-7
    with pytest.raises(HostError, match="needs 16 primes"):
        h.inv_sqrt(h.encrypt(x, DELTA, 15))


@pytest.mark.parametrize("d", [5, 8])
def test_layernorm_over_the_hidden_columns(d):
    """LayerNorm of d hidden columns (one per ciphertext; an odd d exercises the batch sum's
    carried member): mean and variance over the batch, the reference's inverse square root,
    gamma and beta per column; decryptions equal numpy's run of the same arithmetic;
    2 (4 + 2) + 8 = 20 levels."""
    h = _host(bits=[51] + [46] * 19 + [51] + [51] * 5)
    rng = np.random.default_rng(10 + d)
    n = h.n // 2
    z = rng.standard_normal((d, n))
    z = (z - z.mean(axis=0)) / z.std(axis=0)  # per slot: mean 0, variance 1 over the columns
    sigma = rng.uniform(2.0, 20.0, n)  # so that var = sigma^2 lies in [4, 400], inside the guess's range
    x = rng.uniform(-3, 3, n) + sigma * z
    gamma, beta = rng.uniform(0.5, 1.5, d), rng.uniform(-0.5, 0.5, d)
    out = h.layernorm(h.encrypt(x, DELTA, 21), gamma, beta)
    mean = x.mean(axis=0)
    var = ((x - mean) ** 2).mean(axis=0)
    want = gamma[:, None] * (x - mean) * _inv_sqrt_reference(var) + beta[:, None]
    assert out.count == d and out.level == 1 and out.scale == DELTA
    assert np.abs(h.decrypt(out).real - want).max() < 1e-5
    with pytest.raises(HostError, match="needs 21 primes"):
        h.layernorm(h.encrypt(x, DELTA, 20), gamma, beta)


def test_softmax_over_the_batch():
    """softmax over 6 ciphertexts: the reference's exp, a batch sum scaled into (0, 2), its
    Goldschmidt inverse and the product; decryptions equal numpy's run of the same formulas."""
    h = _host(bits=[51] + [46] * 19 + [51] + [51] * 5)
    rng = np.random.default_rng(12)
    x = rng.uniform(-2.0, 2.0, (6, h.n // 2))
    shift, sum_scale, it = 0.5, 1.0 / 32.0, 7
    out = h.softmax(h.encrypt(x, DELTA, 21), shift, sum_scale, it)
    e = (1 + (x - shift) / 128) ** 128
    s = sum_scale * e.sum(axis=0)
    y, r = 1 - s, 2 - s
    for _ in range(it):
        y = y * y
        r = r * (1 + y)
    want = sum_scale * e * r
    assert out.count == 6 and out.level == 21 - it - 12 and out.scale == DELTA
    assert np.abs(h.decrypt(out).real - want).max() < 1e-5
    assert np.abs(want - np.exp(x) / np.exp(x).sum(axis=0)).max() < 0.05  # the formulas approximate softmax
    with pytest.raises(HostError, match="needs 20 primes"):
        h.softmax(h.encrypt(x, DELTA, 19), shift, sum_scale, it)


def _softmax_attention_reference(x, bias, input_num, it):
    """softmax.cuh:119-'s masks and arithmetic on slot vectors."""
    num, slots = x.shape
    nb = slots // 128
    idx = np.arange(slots)

    def selected(i):
        if i == 0:
            return bias == 1
        if input_num < i <= num - input_num:
            return np.zeros(slots, dtype=bool)
        if i <= input_num:
            return (bias == 1) & (idx < nb * (input_num - i))
        return (bias == 1) & (idx >= (num - i) * nb)

    e = []
    for i in range(num):
        sel = selected(i)
        v = x[i] - 8.1 * sel
        e.append((1 + v / 128) ** 128 - np.where(sel, 0.0, 1.0))
    e = np.stack(e)
    s = e.sum(axis=0)
    y, r = 1 - s, 2 - s
    for _ in range(it):
        y = y * y
        r = r * (1 + y)
    return e * r


def test_softmax_attention_is_the_reference_arithmetic():
    """The attention block's softmax with its masks: 6 diagonals, input_num 2, valid token
    slots marked by bias_vec (padding slots hold 0); decryptions equal numpy's run of the
    reference's masks and formulas; iter + 10 levels."""
    h = _host(bits=[51] + [46] * 23 + [51] + [51] * 5)
    rng = np.random.default_rng(13)
    slots, num, it = h.n // 2, 6, 13
    bias = (np.arange(slots) < 1500).astype(np.int32)
    # scores in [0, 0.05] keep every slot's sum in (0, 2), where the inverse converges
    x = np.where(bias == 1, rng.uniform(0.0, 0.05, (num, slots)), 0.0)
    out = h.softmax_attention(h.encrypt(x, DELTA, 25), bias, 2, it)
    assert out.count == num and out.level == 25 - it - 10
    want = _softmax_attention_reference(x, bias, 2, it)
    err = np.abs(h.decrypt(out).real - want)
    assert err[:, bias == 1].max() < 1e-6
    # padding slots: their sum is 0, so the inverse is 2^(iter + 1) and scales the noise of
    # values that are 0 (the reference's caller masks these slots out)
    assert err[:, bias == 0].max() < 1e-3
    with pytest.raises(HostError, match="needs 24 primes"):
        h.softmax_attention(h.encrypt(x, DELTA, 23), bias, 2, it)


def test_polynomial_operators_refuse_bad_inputs(small):
    h = small
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, (2, 16))
    with pytest.raises(HostError, match="not enough levels"):
        h.gelu(h.encrypt(x, DELTA, 6))
    with pytest.raises(HostError, match="not enough levels"):
        h.chebyshev(h.encrypt(x, DELTA, 4), np.ones(6), -1.0, 1.0)
    with pytest.raises(HostError, match="lo < hi"):
        h.chebyshev(h.encrypt(x, DELTA, 6), [0.5, 1.0], 1.0, 1.0)
    with pytest.raises(HostError, match="degree 0"):
        h.chebyshev(h.encrypt(x, DELTA, 6), [0.5], -1.0, 1.0)


@pytest.mark.gpu
def test_cuda_polynomial_operators_match_oracle_build():
    import shmoai_b200.host as H

    g, c = _host(lib=H.PRODUCT_LIB, seed=21), _host(seed=21)
    rng = np.random.default_rng(5)
    x = rng.uniform(-19.5, 12.5, (3, g.n // 2))
    for h_cu, h_or in ((g, c),):
        a, b = h_cu.encrypt(x, DELTA, 9), h_or.encrypt(x, DELTA, 9)
        assert np.array_equal(a.to_host(), b.to_host())
        assert np.array_equal(h_cu.gelu(a).to_host(), h_or.gelu(b).to_host())
        coeffs = rng.uniform(-1, 1, 13)
        assert np.array_equal(h_cu.chebyshev(a, coeffs, -20.0, 13.0).to_host(),
                              h_or.chebyshev(b, coeffs, -20.0, 13.0).to_host())
        assert np.array_equal(h_cu.inverse(h_cu.encrypt(x / 20.0 + 1.0, DELTA, 9), 6).to_host(),
                              h_or.inverse(h_or.encrypt(x / 20.0 + 1.0, DELTA, 9), 6).to_host())
        e1, e2 = h_cu.encrypt(x / 4.0, DELTA, 10), h_or.encrypt(x / 4.0, DELTA, 10)
        assert np.array_equal(h_cu.exp(e1).to_host(), h_or.exp(e2).to_host())
        v1, v2 = h_cu.encrypt(x * 20.0 + 400.0, DELTA, 12), h_or.encrypt(x * 20.0 + 400.0, DELTA, 12)
        assert np.array_equal(h_cu.inv_sqrt(v1, 2, 1).to_host(), h_or.inv_sqrt(v2, 2, 1).to_host())
        z = rng.standard_normal((3, g.n // 2))
        cols = 5.0 * (z - z.mean(axis=0)) / z.std(axis=0)
        w1, w2 = h_cu.encrypt(cols, DELTA, 16), h_or.encrypt(cols, DELTA, 16)
        gm, bt = [1.0, 0.5, 2.0], [0.0, 0.25, -0.5]
        assert np.array_equal(h_cu.layernorm(w1, gm, bt, 2, 1).to_host(), h_or.layernorm(w2, gm, bt, 2, 1).to_host())
        s1, s2 = h_cu.encrypt(x / 10.0, DELTA, 19), h_or.encrypt(x / 10.0, DELTA, 19)
        assert np.array_equal(h_cu.softmax(s1, 0.5, 1.0 / 8.0, 5).to_host(), h_or.softmax(s2, 0.5, 1.0 / 8.0, 5).to_host())


@pytest.mark.gpu
def test_gelu_reference_parameters_on_b200():
    """N = 2^16, the bootstrapping chain, scale 2^46, input at 12 primes, 4 full ciphertexts."""
    import shmoai_b200.host as H

    h = _host(lib=H.PRODUCT_LIB, seed=7, log_n=16, bits=REF_BITS, hw=192)
    rng = np.random.default_rng(6)
    x = rng.uniform(-19.5, 12.5, (4, h.n // 2))
    out = h.gelu(h.encrypt(x, DELTA, 12))
    y = h.decrypt(out).real
    series = np.polynomial.chebyshev.chebval((x + 3.5) / 16.0, GELU_D)
    assert out.level == 6
    assert np.abs(y - series).max() < 1e-5
    assert np.abs(y - _gelu(x)).max() < 0.04


@pytest.mark.gpu
def test_gelu_graph_replay_equals_eager():
    """shm_host_chebyshev_capture: one CUDA graph of the GELU; a launch after writing the next
    batch into the captured input gives that batch's eager result bit for bit."""
    import shmoai_b200.host as H

    h = _host(lib=H.PRODUCT_LIB, seed=31)
    rng = np.random.default_rng(7)
    x1, x2 = (rng.uniform(-19.5, 12.5, (2, h.n // 2)) for _ in range(2))
    a = h.encrypt(x1, DELTA, 9)
    nxt = h.encrypt(x2, DELTA, 9).to_host()
    graph, out = h.capture_chebyshev(a)
    assert graph.kernels > 0
    graph.launch()
    assert np.array_equal(out.to_host(), h.gelu(a).to_host())
    a.write_from_ptr(nxt.ctypes.data)
    graph.launch()
    assert np.array_equal(out.to_host(), h.gelu(a).to_host())
    coeffs = rng.uniform(-1, 1, 9)
    g2, o2 = h.capture_chebyshev(a, coeffs, -20.0, 13.0)
    g2.launch()
    assert np.array_equal(o2.to_host(), h.chebyshev(a, coeffs, -20.0, 13.0).to_host())
