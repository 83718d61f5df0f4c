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
