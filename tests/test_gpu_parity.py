"""CUDA path vs the reference: every golden record reproduced bit for bit by
the C-ABI entry points on a B200, at N = 2^12 and at the full N = 2^16
parameter sets; batched calls vs the CPU oracle."""
import numpy as np
import pytest
import torch

from golden.golden import GoldenSet
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SETS = ["tiny", "prim", "boot"]


@pytest.fixture(scope="module", params=SETS)
def env(request):
    from shmoai_b200.ckks import CKKSContext, to_device

    g = GoldenSet(request.param)
    ctx = CKKSContext(g.log_n, primes=g.primes, n_special=g.np)
    d = {
        "A": to_device(g.ct(1)), "B": to_device(g.ct(2)), "C": to_device(g.plain(3)),
        "rk": to_device(g.relin_key()), "gk5": to_device(g.galois_key(5)),
        "gkc": to_device(g.galois_key(2 * g.n - 1)),
        "D": to_device(g.ct(4, g.L - 1)), "E": to_device(g.ct(5, g.L - 1)),
    }
    yield g, ctx, d
    ctx.close()
    torch.cuda.empty_cache()


def check(g, name, t):
    from shmoai_b200.ckks import to_host

    torch.cuda.synchronize()
    ok, msg = g.matches(name, to_host(t))
    assert ok, msg


def test_context_primes_match_reference(env):
    g, ctx, _ = env
    assert np.array_equal(ctx.primes, g.primes)
    assert ctx.dnum == g.dnum


def test_ntt_inverse(env):
    g, ctx, d = env
    check(g, "intt_A", ctx.ntt_inverse_(d["A"].clone()))


def test_ntt_forward(env):
    g, ctx, d = env
    check(g, "ntt_A", ctx.ntt_forward_(d["A"].clone()))


def test_ntt_round_trip(env):
    _, ctx, d = env
    t = ctx.ntt_forward_(ctx.ntt_inverse_(d["A"].clone()))
    assert torch.equal(t, d["A"])


def test_add_and_multiply_plain(env):
    g, ctx, d = env
    check(g, "add_AB", ctx.add(d["A"], d["B"]))
    check(g, "mulplain_AC", ctx.multiply_plain(d["A"], d["C"]))


def test_rescale(env):
    g, ctx, d = env
    check(g, "rescale_A", ctx.rescale(d["A"]))


def test_rotate_by_one(env):
    g, ctx, d = env
    check(g, "rot1_A", ctx.rotate(d["A"], 1, d["gk5"]))


def test_conjugate(env):
    g, ctx, d = env
    check(g, "conj_A", ctx.apply_galois(d["A"], 2 * g.n - 1, d["gkc"]))


def test_multiply_relinearize_rescale(env):
    g, ctx, d = env
    m = ctx.multiply(d["A"], d["B"])
    check(g, "mul_AB", m)
    r = ctx.relinearize(m, d["rk"])
    check(g, "relin_AB", r)
    check(g, "mrr_AB", ctx.rescale(r))


def test_relinearize_in_place(env):
    g, ctx, d = env
    m = ctx.multiply(d["A"], d["B"])
    ctx.relinearize(m, d["rk"], out=m)
    check(g, "relin_AB", m[:2].contiguous())


def test_lower_level_short_digit(env):
    g, ctx, d = env
    check(g, "rot1_D", ctx.rotate(d["D"], 1, d["gk5"]))
    check(g, "relin_DE", ctx.relinearize(ctx.multiply(d["D"], d["E"]), d["rk"]))


def test_ctpt_matmul(env):
    from shmoai_b200.ckks import to_device

    g, ctx, _ = env
    W = g.ctpt_weights()
    X = to_device(g.ctpt_inputs())
    Y = ctx.ctpt_matmul(X, torch.from_numpy(W).cuda())
    for k in range(W.shape[1]):
        check(g, f"ctpt_sum_{k}", Y[k])
        check(g, f"ctpt_out_{k}", ctx.rescale(Y[k]))


def test_batched_rotate_matches_oracle():
    """n_cts ciphertexts at several levels through one call vs the oracle one by one."""
    from shmoai_b200.ckks import CKKSContext, to_device, to_host

    g = GoldenSet("tiny")
    ctx = CKKSContext(g.log_n, primes=g.primes, n_special=g.np)
    o = O.Oracle(g.log_n, g.primes, g.nq, g.np)
    key = g.galois_key(5)
    for L in range(1, g.L + 1):
        X = np.stack([g.ct(500 + 10 * L + i, L) for i in range(5)])
        Y = to_host(ctx.rotate(to_device(X), 1, to_device(key)))
        for i in range(5):
            assert np.array_equal(Y[i], o.apply_galois_ct(np.ascontiguousarray(X[i]), 5, key)), (L, i)
    ctx.close()


def test_batched_relinearize_matches_oracle():
    from shmoai_b200.ckks import CKKSContext, to_device, to_host

    g = GoldenSet("tiny")
    ctx = CKKSContext(g.log_n, primes=g.primes, n_special=g.np)
    o = O.Oracle(g.log_n, g.primes, g.nq, g.np)
    key = g.relin_key()
    for L in (2, 5, 6):
        X = np.stack([np.concatenate([g.ct(700 + i, L), g.ct(800 + i, L)[:1]]) for i in range(3)])
        Y = to_host(ctx.relinearize(to_device(X), to_device(key)))
        for i in range(3):
            assert np.array_equal(Y[i], o.relinearize(np.ascontiguousarray(X[i]), key)), (L, i)
    ctx.close()


def test_errors_are_reported_not_thrown():
    from shmoai_b200._lib import ShmError
    from shmoai_b200.ckks import CKKSContext

    g = GoldenSet("tiny")
    ctx = CKKSContext(g.log_n, primes=g.primes, n_special=g.np)
    t = torch.zeros(2, g.nq + g.np + 1, g.n, dtype=torch.int64, device="cuda")
    with pytest.raises(ShmError):
        ctx.ntt_forward_(t)  # more limbs than the chain holds
    with pytest.raises(ShmError):
        ctx.rescale(torch.zeros(2, g.nq + 1, g.n, dtype=torch.int64, device="cuda"))  # key level
    with pytest.raises(ValueError):
        ctx.galois_elt(g.n)  # step too large
    ctx.close()


def test_hoisted_rotations_match_oracle():
    """One ModUp, several Galois elements: equal to the oracle's hoisted restatement
    bit for bit, and decrypting like the plain rotation (same message, tiny noise)."""
    from shmoai_b200.ckks import CKKSContext, to_device, to_host

    g = GoldenSet("tiny")
    ctx = CKKSContext(g.log_n, primes=g.primes, n_special=g.np)
    o = O.Oracle(g.log_n, g.primes, g.nq, g.np)
    elts = [5, 25, 2 * g.n - 1, pow(5, 7, 2 * g.n)]
    keys = [g.key(1000 + 10 * i) for i in range(len(elts))]
    for L in (2, 5, 6):
        X = np.stack([g.ct(900 + L * 10 + i, L) for i in range(3)])
        outs = ctx.apply_galois_hoisted(to_device(X), elts, [to_device(k) for k in keys])
        for i in range(3):
            want = o.apply_galois_hoisted(np.ascontiguousarray(X[i]), elts, keys)
            for e in range(len(elts)):
                assert np.array_equal(to_host(outs[e])[i], want[e]), (L, i, e)
    ctx.close()
