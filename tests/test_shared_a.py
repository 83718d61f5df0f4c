"""Shared-a (multi-secret RLWE) batches: FmtSwitch forward / backward, Sh-Rot and
the shared-a S2C-first bootstrap.

CPU: the oracle restatement and the key generation are checked by decryption
(forward then decrypt with the auxiliary secrets s'_i, Sh-Rot then decrypt,
backward then decrypt with s), as the reference's stage probes and
shared_a_fmt_switch_test do (src/include/test/bootstrapping/test_shared_a.cuh:33-248,
1499-1510), and the whole shared-a bootstrap runs on the oracle at N = 2^12.
GPU: the CUDA entry points equal the oracle bit for bit on random groups and keys,
the CUDA shared-a bootstrap equals the oracle's, and the reference parameter set
(N = 2^16, n = 4) meets the decryption-error target.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle_backend import OracleBackend
from shmoai_b200.bootstrap import Bootstrapper
from shmoai_b200.evaluator import Ct, Evaluator, ShCt
from shmoai_b200.keygen import KeyGenerator

SMALL_BITS = [51] + [46] * 6 + [51] * 13 + [51] * 5  # N = 2^12, nq = 20, np = 5 (dnum 4)
REF_BITS = [51] + [46] * 20 + [51] * 14 + [51] * 5


def _setup(n_mem, steps, seed=2):
    be = OracleBackend(12, SMALL_BITS, 5)
    kg = KeyGenerator(be, hamming_weight=64, seed=seed)
    ev = Evaluator(be)
    kg.aux_secrets(n_mem, hamming_weight=64)
    ev.shared.fmt = kg.format_key()
    ev.shared.backward = kg.backward_keys()
    for st in steps:
        e = ev.galois_elt(st)
        ev.shared.galois[e] = kg.shared_galois_key(e)
    return be, kg, ev


@pytest.fixture(scope="module")
def small3():
    return _setup(3, [1, 7, 0])


def _inputs(be, kg, n_cts, L, seed):
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1, 1, (n_cts, be.n // 2)) + 1j * rng.uniform(-1, 1, (n_cts, be.n // 2))
    return z, kg.encrypt(z, 2.0 ** 40, L)


def test_fmt_forward_backward_roundtrip_on_oracle(small3):
    be, kg, ev = small3
    z, ct = _inputs(be, kg, 6, 4, 1)
    sh = ev.to_shared(ct, 3)
    assert isinstance(sh, ShCt) and sh.data.shape == (2, 4, 4, be.n)
    assert np.abs(kg.decrypt_shared(sh.data, sh.scale) - z).max() < 1e-6
    back = ev.from_shared(sh)
    assert back.data.shape == ct.data.shape
    assert np.abs(kg.decrypt(back) - z).max() < 1e-6


def test_sh_rotate_and_conjugate_on_oracle(small3):
    be, kg, ev = small3
    z, ct = _inputs(be, kg, 3, 5, 2)
    sh = ev.to_shared(ct, 3)
    rot = ev.rotate_many(sh, [1, 7])
    for st, r in rot.items():
        assert isinstance(r, ShCt)
        assert np.abs(kg.decrypt_shared(r.data, r.scale) - np.roll(z, -st, axis=1)).max() < 1e-6
    cj = ev.conjugate(sh)
    assert np.abs(kg.decrypt_shared(cj.data, cj.scale) - np.conj(z)).max() < 1e-6


def test_shared_ops_keep_the_group_form(small3):
    be, kg, ev = small3
    z, ct = _inputs(be, kg, 3, 5, 3)
    sh = ev.to_shared(ct, 3)
    s2 = ev.mul_i(ev.add(sh, sh))
    assert isinstance(s2, ShCt)
    assert np.abs(kg.decrypt_shared(s2.data, s2.scale) - 2j * z).max() < 1e-6
    with pytest.raises(TypeError):
        ev.add_const(sh, 1.0)
    with pytest.raises(ValueError):
        ev.rotate(sh, 3)  # no Sh-Galois key for this step


def test_shared_bootstrap_on_oracle():
    be = OracleBackend(12, SMALL_BITS, 5)
    kg = KeyGenerator(be, hamming_weight=64, seed=4)
    ev = Evaluator(be)
    ev.relin_key = kg.relin_key()
    bs = Bootstrapper(ev)
    kg.aux_secrets(2, hamming_weight=64)
    ev.shared.fmt = kg.format_key()
    ev.shared.backward = kg.backward_keys()
    for elt in bs.galois_elts():
        ev.shared.galois[elt] = kg.shared_galois_key(elt)
    rng = np.random.default_rng(6)
    n = be.n // 2
    z = rng.uniform(-1, 1, (2, n)) + 1j * rng.uniform(-1, 1, (2, n))
    ct = kg.encrypt(z, 2.0 ** 46, 4)
    out = bs.bootstrap_shared(ct, 2)
    err = np.abs(kg.decrypt(out) - z)
    assert out.level == 20 - 3 - 9 and out.batch == 2
    assert err.mean() < 2e-5, err.mean()
    assert err.max() < 1e-4, err.max()


# ------------------------------------------------------------------ GPU parity


def _rand(rng, shape, primes_rows):
    out = np.empty(shape, dtype=np.uint64)
    for i, q in enumerate(primes_rows):
        out[..., i, :] = rng.integers(0, q, size=shape[:-2] + (shape[-1],), dtype=np.uint64)
    return out


def _qp_rows(o, L):
    return [int(p) for p in o.primes[:L]]


@pytest.mark.gpu
@pytest.mark.parametrize("set_name,G,n_mem,L", [("tiny", 2, 3, 3), ("tiny", 1, 4, 6), ("boot", 1, 4, 4)])
def test_shared_entry_points_match_oracle(set_name, G, n_mem, L):
    from shmoai_b200.backend import GpuBackend
    from shmoai_b200.ckks import CKKSContext

    log_n, bits, n_sp = O.PARAM_SETS[set_name]
    o = O.Oracle.from_bits(log_n, bits, n_sp)
    N, QP = o.n, o.nq + o.np
    qp = [int(p) for p in o.primes]
    rng = np.random.default_rng(100 + L)
    ctx = CKKSContext(log_n, primes=qp, n_special=n_sp)
    gb = GpuBackend(ctx)
    H = n_mem + 1
    sh = _rand(rng, (G, H, L, N), qp[:L])
    elts = [O.galois_elt_from_step(log_n, s) for s in (1, -3)] + [2 * N - 1]
    keys = [_rand(rng, (o.dnum, H, QP, N), qp) for _ in elts]
    got = gb.sh_rotate_many(gb.from_host(sh), elts, [gb.from_host(k) for k in keys])
    for e in range(len(elts)):
        want = np.stack([o.shared_rotate_hoisted(sh[g], elts, keys)[e] for g in range(G)])
        assert np.array_equal(gb.to_host(got[e]), want), f"Sh-Rot elt {elts[e]}"

    cts = _rand(rng, (G * n_mem, 2, L, N), qp[:L])
    fkey = _rand(rng, (n_mem, H, QP, N), qp)
    got = gb.to_host(gb.fmt_forward(gb.from_host(cts), n_mem, gb.from_host(fkey)))
    want = np.stack([o.fmt_forward(cts[g * n_mem:(g + 1) * n_mem], fkey) for g in range(G)])
    assert np.array_equal(got, want), "FmtSwitch forward"

    bkeys = [_rand(rng, (o.dnum, 2, QP, N), qp) for _ in range(n_mem)]
    got = gb.to_host(gb.fmt_backward(gb.from_host(sh), [gb.from_host(k) for k in bkeys]))
    want = np.concatenate([o.fmt_backward(sh[g], bkeys) for g in range(G)])
    assert np.array_equal(got, want), "FmtSwitch backward"
    ctx.close()


@pytest.mark.gpu
def test_shared_bootstrap_cuda_matches_oracle_bit_for_bit():
    from shmoai_b200.backend import GpuBackend
    from shmoai_b200.ckks import CKKSContext

    be = OracleBackend(12, SMALL_BITS, 5)
    kg = KeyGenerator(be, hamming_weight=64, seed=8)
    ev = Evaluator(be)
    ev.relin_key = kg.relin_key()
    bs = Bootstrapper(ev)
    kg.aux_secrets(2, hamming_weight=64)
    ev.shared.fmt = kg.format_key()
    ev.shared.backward = kg.backward_keys()
    for elt in bs.galois_elts():
        ev.shared.galois[elt] = kg.shared_galois_key(elt)
    rng = np.random.default_rng(9)
    n = be.n // 2
    z = rng.uniform(-1, 1, (4, n)) + 1j * rng.uniform(-1, 1, (4, n))
    ct = kg.encrypt(z, 2.0 ** 46, 4)
    ref = bs.bootstrap_shared(ct, 2)

    ctx = CKKSContext(12, primes=be.primes, n_special=5)
    gb = GpuBackend(ctx)
    gev = Evaluator(gb, relin_key=gb.from_host(ev.relin_key))
    gev.shared.fmt = gb.from_host(ev.shared.fmt)
    gev.shared.backward = [gb.from_host(k) for k in ev.shared.backward]
    gev.shared.galois = {e: gb.from_host(k) for e, k in ev.shared.galois.items()}
    out = Bootstrapper(gev).bootstrap_shared(Ct(gb.from_host(ct.data), ct.scale), 2)
    assert out.level == ref.level and out.scale == ref.scale
    assert np.array_equal(gb.to_host(out.data), ref.data)
    ctx.close()


@pytest.mark.gpu
def test_shared_bootstrap_reference_parameters_on_b200():
    """N = 2^16, the reference's parameters, n = 4 members per group, 8 ciphertexts."""
    import torch

    from shmoai_b200.backend import GpuBackend
    from shmoai_b200.ckks import CKKSContext

    ctx = CKKSContext(16, bits=REF_BITS, n_special=5)
    be = GpuBackend(ctx)
    kg = KeyGenerator(be, hamming_weight=192, seed=12)
    ev = Evaluator(be, relin_key=kg.relin_key())
    bs = Bootstrapper(ev)
    kg.aux_secrets(4, hamming_weight=192)
    ev.shared.fmt = kg.format_key()
    ev.shared.backward = kg.backward_keys()
    for elt in bs.galois_elts():
        ev.shared.galois[elt] = kg.shared_galois_key(elt)
    rng = np.random.default_rng(13)
    n = be.n // 2
    z = rng.uniform(-1, 1, (8, n)) + 1j * rng.uniform(-1, 1, (8, n))
    ct = kg.encrypt(z, 2.0 ** 46, 4)
    out = bs.bootstrap_shared(ct, 4)
    torch.cuda.synchronize()
    err = np.abs(kg.decrypt(out) - z)
    print(f"shared-a bootstrap N=2^16 n=4: level {out.level}, mean |err| {err.mean():.3e}, max {err.max():.3e}")
    assert out.level == 35 - 3 - 9
    assert err.mean() < 2e-5, err.mean()
    assert err.max() < 2e-4, err.max()
    ctx.close()
