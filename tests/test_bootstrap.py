"""S2C-first bootstrapping: the slot-transform factorisation, the pipeline on
the CPU oracle (N = 2^12), the CUDA pipeline bit for bit against the oracle
pipeline with the same keys, and the full reference parameter set (N = 2^16)
on a B200 judged by decryption error (the reference's own criterion: mean
|err| over slots, README 1.33e-5; target 2e-5)."""
import numpy as np
import pytest

from oracle_backend import OracleBackend
from shmoai_b200.bootstrap import Bootstrapper, apply_diags, c2s_layers, cheb_divide, s2c_layers
from shmoai_b200.encoder import Encoder
from shmoai_b200.evaluator import Ct, Evaluator
from shmoai_b200.keygen import KeyGenerator

SMALL_BITS = [51] + [46] * 6 + [51] * 13 + [51] * 5  # N = 2^12, nq = 20, np = 5 (dnum 4)
REF_BITS = [51] + [46] * 20 + [51] * 14 + [51] * 5  # test_shared_a.cuh:1208-1250


def bitrev_perm(n):
    b = n.bit_length() - 1
    return np.array([int(format(i, f"0{b}b")[::-1], 2) for i in range(n)])


@pytest.mark.parametrize("log_n", [6, 9, 12])
def test_slot_transform_factorisation(log_n):
    N = 1 << log_n
    n = N // 2
    enc = Encoder(log_n)
    omega = np.exp(2j * np.pi * enc.exps / (2 * N))
    rng = np.random.default_rng(log_n)
    w = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    Vw = np.array([np.sum(w * o ** np.arange(n)) for o in omega])
    y = w[bitrev_perm(n)]
    for layer in s2c_layers(n):
        y = apply_diags(layer, y)
    assert np.abs(y - Vw).max() < 1e-9 * np.abs(Vw).max()
    z = Vw
    for layer in c2s_layers(n):
        z = apply_diags(layer, z)
    assert np.abs(z - w[bitrev_perm(n)]).max() < 1e-9


def test_chebyshev_division():
    from numpy.polynomial import chebyshev as C

    c = np.random.default_rng(0).standard_normal(48)
    q, r = cheb_divide(c, 32)
    x = np.linspace(-1, 1, 11)
    assert np.allclose(C.chebval(x, c), C.chebval(x, q) * C.chebval(x, [0] * 32 + [1]) + C.chebval(x, r))


def _small_setup(seed=1):
    be = OracleBackend(12, SMALL_BITS, 5)
    kg = KeyGenerator(be, hamming_weight=64, seed=seed)
    ev = Evaluator(be)
    ev.relin_key = kg.relin_key()
    bs = Bootstrapper(ev)
    for elt in bs.galois_elts():
        ev.galois_keys[elt] = kg.galois_key(elt)
    return be, kg, ev, bs


@pytest.fixture(scope="module")
def small():
    return _small_setup()


def test_bootstrap_on_oracle(small):
    be, kg, ev, bs = small
    rng = np.random.default_rng(3)
    n = be.n // 2
    z = rng.uniform(-1, 1, (2, n)) + 1j * rng.uniform(-1, 1, (2, n))
    ct = kg.encrypt(z, 2.0 ** 46, 4)
    out = bs.bootstrap(ct)
    err = np.abs(kg.decrypt(out) - z)
    assert out.level == 20 - 3 - 9
    assert abs(out.scale - 2.0 ** 46) < 1e-6 * 2.0 ** 46
    assert err.mean() < 2e-5, err.mean()
    assert err.max() < 1e-4, err.max()


@pytest.mark.gpu
def test_bootstrap_cuda_matches_oracle_bit_for_bit(small):
    """The whole pipeline on the CUDA library with the oracle's keys and input
    produces the oracle pipeline's output limbs exactly."""
    from shmoai_b200.backend import GpuBackend
    from shmoai_b200.ckks import CKKSContext

    be, kg, ev, bs = small
    rng = np.random.default_rng(5)
    n = be.n // 2
    z = rng.uniform(-1, 1, (2, n)) + 1j * rng.uniform(-1, 1, (2, n))
    ct = kg.encrypt(z, 2.0 ** 46, 4)
    ref = bs.bootstrap(ct)

    ctx = CKKSContext(12, primes=be.primes, n_special=5)
    gb = GpuBackend(ctx)
    gev = Evaluator(gb, relin_key=gb.from_host(ev.relin_key),
                    galois_keys={e: gb.from_host(k) for e, k in ev.galois_keys.items()})
    gbs = Bootstrapper(gev)
    out = gbs.bootstrap(Ct(gb.from_host(ct.data), ct.scale))
    assert out.level == ref.level and out.scale == ref.scale
    assert np.array_equal(gb.to_host(out.data), ref.data)
    ctx.close()


@pytest.mark.gpu
def test_bootstrap_reference_parameters_on_b200():
    """N = 2^16, Q = [51] + 20x[46] + 14x[51], P = 5x[51], Delta = 2^46, h = 192,
    input at 4 primes, full 2^15 slots uniform in [-1, 1]^2."""
    import torch

    from shmoai_b200.backend import GpuBackend
    from shmoai_b200.ckks import CKKSContext

    ctx = CKKSContext(16, bits=REF_BITS, n_special=5)
    be = GpuBackend(ctx)
    kg = KeyGenerator(be, hamming_weight=192, seed=7)
    ev = Evaluator(be, relin_key=kg.relin_key())
    bs = Bootstrapper(ev)
    for elt in bs.galois_elts():
        ev.galois_keys[elt] = kg.galois_key(elt)
    rng = np.random.default_rng(11)
    n = be.n // 2
    z = rng.uniform(-1, 1, (2, n)) + 1j * rng.uniform(-1, 1, (2, n))
    ct = kg.encrypt(z, 2.0 ** 46, 4)
    out = bs.bootstrap(ct)
    torch.cuda.synchronize()
    err = np.abs(kg.decrypt(out) - z)
    print(f"bootstrap N=2^16: level {out.level}, mean |err| {err.mean():.3e}, max {err.max():.3e}")
    assert out.level == 35 - 3 - 9
    assert err.mean() < 2e-5, err.mean()
    assert err.max() < 2e-4, err.max()
    ctx.close()
