"""Shared-a primitives and the slot-vector encoder against the reference's own outputs.

The fixtures ``golden_shared_<set>.json`` come from the reference's FmtSwitch.cu, ShRotate.cu,
SharedABatchOps.cu and PhantomCKKSEncoder (ckks.cu:89-187) built for sm_100a and run on a
B200 (oracle/ref_golden.cu, mode ``shared``; tests/golden/make_golden.py).  The oracle is
checked against them on the CPU; the CUDA entry points are checked against them on the GPU.
Integer records are compared bit for bit.  The encoder is FP64: its integer coefficients must
equal the reference's except where the exact coefficient lies within the FP64 transforms' error
of a rounding tie (checked in extended precision)."""
import numpy as np
import pytest

from golden.golden import SharedGoldenSet, exact_coefficient
from oracle import oracle as O

SETS = ["tiny", "boot"]


def _fmt_cases(g):
    return [(int(k.split("_")[2][1:]), int(k.split("_")[3][1:])) for k in g.doc if k.startswith("fmt_fwd_")]


def _rot_cases(g):
    out = []
    for k in g.doc:
        if k.startswith("shrot_") and not k.endswith("_elt"):
            _, n, L, s = k.split("_")
            out.append((k, int(n[1:]), int(L[1:]), int(g.doc[k + "_elt"])))
    return out


@pytest.fixture(scope="module", params=SETS)
def gset(request):
    g = SharedGoldenSet(request.param)
    return g, O.Oracle(g.log_n, g.primes, g.nq, g.np)


def _check(g, name, arr):
    ok, msg = g.matches(name, arr)
    assert ok, msg


def test_oracle_fmt_switch_matches_reference(gset):
    g, o = gset
    for n, L in _fmt_cases(g):
        _check(g, f"fmt_fwd_n{n}_L{L}", o.fmt_forward(g.cts(30, n, L), g.fmt_key(n, L)))
        _check(g, f"fmt_bwd_n{n}_L{L}", o.fmt_backward(g.batch(50, n, L), g.backward_keys(n)))


def test_oracle_shared_rotate_matches_reference(gset):
    """Sh-Rot in the reference's order (automorphism, then ModUp of the rotated a) equals the reference; the
    hoisted form (ModUp first, automorphism on the extended digits) decrypts the same but differs in the
    limbs by the base conversion's overflow multiples, so it is not the reference's bits."""
    g, o = gset
    for name, n, L, elt in _rot_cases(g):
        _check(g, name, o.shared_rotate(g.batch(60, n, L), elt, g.shrot_key(n)))
    name, n, L, elt = _rot_cases(g)[0]
    hoisted = o.shared_rotate_hoisted(g.batch(60, n, L), [elt], [g.shrot_key(n)])[0]
    assert not g.matches(name, hoisted)[0]


def test_oracle_shared_batch_ops_match_reference(gset):
    g, o = gset
    n = 4
    _check(g, "shared_rescale", o.rescale(g.batch(70, n, g.nq - 1)))
    _check(g, "shared_modraise", o.modraise(g.batch(80, n, 1), g.nq))
    _check(g, "shared_mulplain", o.multiply_plain(g.batch(90, n, 3), g.plain_at(98, 3)))
    _check(g, "shared_add", o.add(g.batch(110, n, 3), g.batch(120, n, 3)))


def _encode_agreement(g, ours: np.ndarray):
    """Coefficients of this library's encode against the reference's: equal, or (rarely) one apart where
    the exact value is within 1e-2 of a rounding tie."""
    scale, stride, ref = g.encode_coeffs()
    mine = ours[::stride]
    diff = mine - ref
    assert np.abs(diff).max(initial=0) <= 1
    bad = np.flatnonzero(diff)
    assert len(bad) <= max(2, len(ref) // 1000), f"{len(bad)} of {len(ref)} coefficients differ"
    z = g.slots()
    for i in bad:
        x = exact_coefficient(z, int(i) * stride, scale, g.log_n)
        assert abs(abs(x - np.floor(x)) - 0.5) < 1e-2, f"coefficient {i * stride}: {mine[i]} vs {ref[i]}, exact {x!r}"
    return len(bad), len(ref)


def test_host_encoder_matches_reference_encode(gset):
    """The host library's FP64 encoder (oracle build: the host FFT restatement) against the reference's."""
    import os

    from shmoai_b200.host import Host

    g, _ = gset
    lib = os.path.join(os.path.dirname(O.HERE), "oracle", "_build", "libshmoai_host_oracle.so")
    h = Host(g.log_n, [int(p) for p in g.primes], g.np, hamming_weight=64, seed=1, lib=lib)
    scale, _, _ = g.encode_coeffs()
    _encode_agreement(g, h.encode_coeffs(g.slots(), scale, on_host=True))
    h.close()


@pytest.mark.gpu
def test_cuda_shared_entry_points_match_reference(gset):
    from shmoai_b200.ckks import CKKSContext, to_device, to_host

    g, _ = gset
    ctx = CKKSContext(g.log_n, primes=[int(p) for p in g.primes], n_special=g.np)
    dev = to_device
    for n, L in _fmt_cases(g):
        got = to_host(ctx.fmt_forward(dev(g.cts(30, n, L)), n, dev(g.fmt_key(n, L))))
        _check(g, f"fmt_fwd_n{n}_L{L}", got)
        got = to_host(ctx.fmt_backward(dev(g.batch(50, n, L)[None]), [dev(k) for k in g.backward_keys(n)]))
        _check(g, f"fmt_bwd_n{n}_L{L}", got)
    for name, n, L, elt in _rot_cases(g):
        got = ctx.shared_rotate(dev(g.batch(60, n, L)[None]), elt, dev(g.shrot_key(n)))
        _check(g, name, to_host(got[0]))
    n = 4
    _check(g, "shared_rescale", to_host(ctx.rescale(dev(g.batch(70, n, g.nq - 1)))))
    _check(g, "shared_modraise", to_host(ctx.modraise(dev(g.batch(80, n, 1)), g.nq)))
    _check(g, "shared_mulplain", to_host(ctx.multiply_plain(dev(g.batch(90, n, 3)), dev(g.plain_at(98, 3)))))
    _check(g, "shared_add", to_host(ctx.add(dev(g.batch(110, n, 3)), dev(g.batch(120, n, 3)))))
    ctx.close()


@pytest.mark.gpu
def test_cuda_encoder_matches_reference_encode(gset):
    """The device encoder (shm_encode) against the reference's; where every compared coefficient is equal,
    the lifted NTT-form plaintext must equal the reference's record bit for bit."""
    from shmoai_b200.host import Host

    g, o = gset
    h = Host(g.log_n, [int(p) for p in g.primes], g.np, hamming_weight=64, seed=1)
    scale, stride, _ = g.encode_coeffs()
    coeffs = h.encode_coeffs(g.slots(), scale)
    n_bad, _ = _encode_agreement(g, coeffs)
    if n_bad == 0 and stride == 1:
        res = np.stack([np.array([int(c) % int(q) for c in coeffs], dtype=np.uint64) for q in g.primes[:g.nq]])
        _check(g, "encode_z", o.ntt(res))
    h.close()
