"""Shared-a (multi-secret RLWE) entry points of the C ABI against the oracle, bit for
bit, on random groups and random keys: Sh-Rot hoisted over several elements
(ShRotate.cu:201-257), FmtSwitch forward with the exact Ql -> P extension
(FmtSwitch.cu:82-108, 276-394) and FmtSwitch backward (FmtSwitch.cu:396-429).
Decryption-level checks of the same operations (and of the keys) run through the
C++ host library in test_host.py."""
import numpy as np
import pytest

from oracle import oracle as O


def _rand(rng, shape, primes_rows):
    out = np.empty(shape, dtype=np.uint64)
    for i, q in enumerate(primes_rows):
        out[..., i, :] = rng.integers(0, q, size=shape[:-2] + (shape[-1],), dtype=np.uint64)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("set_name,G,n_mem,L", [("tiny", 2, 3, 3), ("tiny", 1, 4, 6), ("boot", 1, 4, 4)])
def test_shared_entry_points_match_oracle(set_name, G, n_mem, L):
    from shmoai_b200.ckks import CKKSContext, to_device, to_host

    log_n, bits, n_sp = O.PARAM_SETS[set_name]
    o = O.Oracle.from_bits(log_n, bits, n_sp)
    N, QP = o.n, o.nq + o.np
    qp = [int(p) for p in o.primes]
    rng = np.random.default_rng(100 + L)
    ctx = CKKSContext(log_n, primes=qp, n_special=n_sp)
    H = n_mem + 1
    sh = _rand(rng, (G, H, L, N), qp[:L])
    elts = [O.galois_elt_from_step(log_n, s) for s in (1, -3)] + [2 * N - 1]
    keys = [_rand(rng, (o.dnum, H, QP, N), qp) for _ in elts]
    got = ctx.shared_rotate_hoisted(to_device(sh), elts, [to_device(k) for k in keys])
    for e in range(len(elts)):
        want = np.stack([o.shared_rotate_hoisted(sh[g], elts, keys)[e] for g in range(G)])
        assert np.array_equal(to_host(got[e]), want), f"Sh-Rot elt {elts[e]}"

    cts = _rand(rng, (G * n_mem, 2, L, N), qp[:L])
    fkey = _rand(rng, (n_mem, H, QP, N), qp)
    got = to_host(ctx.fmt_forward(to_device(cts), n_mem, to_device(fkey)))
    want = np.stack([o.fmt_forward(cts[g * n_mem:(g + 1) * n_mem], fkey) for g in range(G)])
    assert np.array_equal(got, want), "FmtSwitch forward"

    bkeys = [_rand(rng, (o.dnum, 2, QP, N), qp) for _ in range(n_mem)]
    got = to_host(ctx.fmt_backward(to_device(sh), [to_device(k) for k in bkeys]))
    want = np.concatenate([o.fmt_backward(sh[g], bkeys) for g in range(G)])
    assert np.array_equal(got, want), "FmtSwitch backward"
    ctx.close()


@pytest.mark.gpu
def test_shared_entry_points_reject_bad_shapes():
    from shmoai_b200._lib import ShmError
    from shmoai_b200.ckks import CKKSContext, to_device

    log_n, bits, n_sp = O.PARAM_SETS["tiny"]
    o = O.Oracle.from_bits(log_n, bits, n_sp)
    ctx = CKKSContext(log_n, primes=[int(p) for p in o.primes], n_special=n_sp)
    N, QP = o.n, o.nq + o.np
    sh = to_device(np.zeros((1, 3, o.nq + 1, N), dtype=np.uint64))  # L above the chain
    key = to_device(np.zeros((o.dnum, 3, QP, N), dtype=np.uint64))
    with pytest.raises(ShmError):
        ctx.shared_rotate_hoisted(sh, [5], [key])
    ctx.close()


def _near_integer_coefficients(primes, L, n, rng):
    """Coefficients x in [0, Q) whose CRT quotient sum  sum_i y_i / q_i = v + x / Q  lies just below
    an integer (x = Q - k for small k), at small x, around Q/2, and random elsewhere."""
    Q = 1
    for q in primes[:L]:
        Q *= int(q)
    xs = [Q - 1 - k for k in range(256)] + list(range(256)) + [Q // 2 + k - 128 for k in range(256)]
    xs += [int.from_bytes(rng.bytes(32), "little") % Q for _ in range(n - len(xs))]
    return xs, Q


def _reference_floor_guard_rows(primes, p_rows, L, xs, Q):
    """FmtSwitch.cu:86-106 in Python floats (IEEE doubles, the reference's operation order): the P rows in
    coefficient form and how many coefficients took the upward guard."""
    qs = [int(q) for q in primes[:L]]
    qhat = [Q // q for q in qs]
    qhat_inv = [pow(qhat[i] % qs[i], -1, qs[i]) for i in range(L)]
    rows = [[0] * len(xs) for _ in p_rows]
    guarded = 0
    for t, x in enumerate(xs):
        ys = [(x % qs[i]) * qhat_inv[i] % qs[i] for i in range(L)]
        frac = 0.0
        for i in range(L):
            frac = frac + float(ys[i]) / float(qs[i])
        v = int(frac)
        if frac - float(v) > 1.0 - 1e-9:
            v += 1
            guarded += 1
        acc = sum(ys[i] * qhat[i] for i in range(L)) - v * Q
        for k, p in enumerate(p_rows):
            rows[k][t] = acc % int(p)
    return rows, guarded


def test_exact_extension_follows_the_reference_floor_guard():
    """The oracle's exact Ql -> P extension equals FmtSwitch.cu:86-106 computed independently (true
    division, limb-order double sum, the 1 - 1e-9 upward guard) on coefficients whose quotient sum sits
    just below an integer, where a reciprocal multiply without the guard floors one too low."""
    log_n, bits, n_sp = O.PARAM_SETS["tiny"]
    o = O.Oracle.from_bits(log_n, bits, n_sp)
    L, n = 3, o.n
    xs, Q = _near_integer_coefficients(o.primes, L, n, np.random.default_rng(7))
    coeff = np.array([[x % int(q) for x in xs] for q in o.primes[:L]], dtype=np.uint64)
    a = o.ntt(coeff)
    ext = o.exact_extend(a)
    assert np.array_equal(ext[:L], a)
    p_rows = [int(p) for p in o.primes[o.nq:]]
    want, guarded = _reference_floor_guard_rows(o.primes, p_rows, L, xs, Q)
    assert guarded > 0, "no coefficient exercised the guard"
    for k, p in enumerate(p_rows):
        single = O.Oracle(log_n, [p], 1, 0)
        got = single.intt(ext[L + k][None])[0]
        assert np.array_equal(got, np.array(want[k], dtype=np.uint64)), f"P row {k}"


@pytest.mark.gpu
def test_fmt_forward_near_integer_quotients_matches_oracle():
    """FmtSwitch forward on the GPU with a-parts whose CRT quotient sums sit just below integers: the
    kernel's extension must take the same upward guard as the oracle (FmtSwitch.cu:86-106)."""
    from shmoai_b200.ckks import CKKSContext, to_device, to_host

    log_n, bits, n_sp = O.PARAM_SETS["tiny"]
    o = O.Oracle.from_bits(log_n, bits, n_sp)
    L, n, n_mem, QP = 3, o.n, 2, o.nq + o.np
    qp = [int(p) for p in o.primes]
    rng = np.random.default_rng(11)
    cts = _rand(rng, (n_mem, 2, L, n), qp[:L])
    for j in range(n_mem):
        xs, _ = _near_integer_coefficients(o.primes, L, n, np.random.default_rng(20 + j))
        cts[j, 1] = o.ntt(np.array([[x % q for x in xs] for q in qp[:L]], dtype=np.uint64))
    fkey = _rand(rng, (n_mem, n_mem + 1, QP, n), qp)
    ctx = CKKSContext(log_n, primes=qp, n_special=n_sp)
    got = to_host(ctx.fmt_forward(to_device(cts), n_mem, to_device(fkey)))
    assert np.array_equal(got, o.fmt_forward(cts, fkey)[None])
    ctx.close()
