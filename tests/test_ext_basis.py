"""The extended basis QlP of the double-hoisted shared-a linear transforms: shm_extend,
shm_add_ext, shm_moddown_ext, shm_multiply_plain_accumulate_ext, shm_lift_signed_ext,
shm_ntt_forward_ext and shm_shared_rotate_ext.

CPU (the oracle's C ABI): the algebra that makes double hoisting exact where it should be —
ModDown(P x) = x, and ModDown of an extended Sh-Rot equals the ordinary Sh-Rot bit for bit,
from an ordinary and from an extended input; the extended encoding's Q limbs are the
ordinary encoding.  GPU: every CUDA entry point against the oracle's, bit for bit.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_CAPI = os.path.join(ROOT, "oracle", "_build", "libshmoai_oracle_capi.so")
LOG_N, BITS, NP = O.PARAM_SETS["tiny"]  # N = 2^12, 6 + 2 primes, dnum 3
P = ctypes.c_void_p
U32 = ctypes.c_uint32
SZ = ctypes.c_size_t


def _bind(lib):
    lib.shm_last_error.restype = ctypes.c_char_p
    sig = {
        "shm_context_create_from_primes": [ctypes.POINTER(P), U32, ctypes.POINTER(ctypes.c_uint64), U32, U32,
                                           ctypes.c_int],
        "shm_context_destroy": [P],
        "shm_extend": [P, P, P, U32, U32, P],
        "shm_add_ext": [P, P, P, P, U32, U32, P],
        "shm_moddown_ext": [P, P, P, U32, U32, P, SZ, P],
        "shm_multiply_plain_accumulate_ext": [P, ctypes.POINTER(P), ctypes.POINTER(P), U32, P, U32, U32,
                                              ctypes.c_int, P],
        "shm_lift_signed_ext": [P, P, P, U32, U32, P],
        "shm_ntt_forward_ext": [P, P, U32, U32, P],
        "shm_lift_signed": [P, P, P, U32, U32, P],
        "shm_ntt_forward": [P, P, U32, U32, P],
        "shm_shared_rotate_ext": [P, P, ctypes.c_int, U32, U32, U32, ctypes.POINTER(U32), ctypes.POINTER(P),
                                  ctypes.POINTER(P), U32, P, SZ, P],
        "shm_shared_rotate_hoisted": [P, P, U32, U32, U32, ctypes.POINTER(U32), ctypes.POINTER(P),
                                      ctypes.POINTER(P), U32, P, SZ, P],
    }
    for name, args in sig.items():
        getattr(lib, name).argtypes = args
    return lib


class Api:
    """One C ABI (the CUDA library on device tensors, or the oracle on host arrays) over the
    same primes; arrays go in and come back as numpy uint64."""

    def __init__(self, lib, primes, device):
        self.lib, self.device = _bind(lib), device
        self.h = P()
        pr = np.ascontiguousarray(primes, dtype=np.uint64)
        rc = self.lib.shm_context_create_from_primes(ctypes.byref(self.h), LOG_N,
                                                     pr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                                     len(pr) - NP, NP, 0)
        assert rc == 0, self.lib.shm_last_error()
        self.keep = []

    def buf(self, a):
        if self.device:
            import torch
            t = torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()
        else:
            t = np.ascontiguousarray(a).copy()
        self.keep.append(t)
        return t

    def ptr(self, t):
        return t.data_ptr() if self.device else t.ctypes.data

    def host(self, t):
        if self.device:
            import torch
            torch.cuda.synchronize()
            return t.cpu().numpy().view(np.uint64)
        return t

    def empty(self, shape):
        return self.buf(np.zeros(shape, dtype=np.uint64))

    def ok(self, rc):
        assert rc == 0, self.lib.shm_last_error()

    def close(self):
        self.lib.shm_context_destroy(self.h)


def _rand(rng, shape, primes_rows):
    out = np.empty(shape, dtype=np.uint64)
    for i, q in enumerate(primes_rows):
        out[..., i, :] = rng.integers(0, q, size=shape[:-2] + (shape[-1],), dtype=np.uint64)
    return out


def _ext_primes(qp, L):
    return qp[:L] + qp[len(qp) - NP:]


def _ops(api, qp, rng, G, n_mem, L):
    """Every extended-basis entry point on one seeded case; returns the outputs by name."""
    N, H, dnum = 1 << LOG_N, n_mem + 1, (len(qp) - NP) // NP
    LP, QP = L + NP, len(qp)
    sh = _rand(rng, (G, H, L, N), qp[:L])
    ext_in = _rand(rng, (G, H, LP, N), _ext_primes(qp, L))
    elts = [O.galois_elt_from_step(LOG_N, s) for s in (1, -3)]
    keys = [_rand(rng, (dnum, H, QP, N), qp) for _ in elts]
    pts = [_rand(rng, (1, LP, N), _ext_primes(qp, L))[0] for _ in range(3)]
    coeffs = rng.integers(-2 ** 40, 2 ** 40, (2, N), dtype=np.int64)
    out = {}
    d_sh, d_ext = api.buf(sh), api.buf(ext_in)
    d_keys = [api.buf(k) for k in keys]
    kp = (P * len(elts))(*[api.ptr(k) for k in d_keys])
    el = (U32 * len(elts))(*elts)
    # rotations: ordinary input, extended input, and the ordinary Sh-Rot for comparison
    for name, src, flag in (("rot_q", d_sh, 0), ("rot_x", d_ext, 1)):
        outs = [api.empty((G, H, LP, N)) for _ in elts]
        op = (P * len(elts))(*[api.ptr(o) for o in outs])
        api.ok(api.lib.shm_shared_rotate_ext(api.h, api.ptr(src), flag, G, n_mem, len(elts), el, kp, op, L, None, 0,
                                             None))
        out[name] = [api.host(o).copy() for o in outs]
    outs = [api.empty((G, H, L, N)) for _ in elts]
    op = (P * len(elts))(*[api.ptr(o) for o in outs])
    api.ok(api.lib.shm_shared_rotate_hoisted(api.h, api.ptr(d_sh), G, n_mem, len(elts), el, kp, op, L, None, 0, None))
    out["rot_plain"] = [api.host(o).copy() for o in outs]
    # extend, add, ModDown
    e = api.empty((G, H, LP, N))
    api.ok(api.lib.shm_extend(api.h, api.ptr(d_sh), api.ptr(e), G * H, L, None))
    out["extend"] = api.host(e).copy()
    s = api.empty((G, H, LP, N))
    api.ok(api.lib.shm_add_ext(api.h, api.ptr(e), api.ptr(d_ext), api.ptr(s), G * H, L, None))
    out["add"] = api.host(s).copy()
    md = api.empty((G, H, L, N))
    api.ok(api.lib.shm_moddown_ext(api.h, api.ptr(s), api.ptr(md), G * H, L, None, 0, None))
    out["moddown"] = api.host(md).copy()
    # multiply-plain-accumulate over QlP
    terms = [api.buf(ext_in), api.buf(out["rot_q"][0]), api.buf(out["rot_x"][1])]
    d_pts = [api.buf(p) for p in pts]
    acc = api.empty((G, H, LP, N))
    api.ok(api.lib.shm_multiply_plain_accumulate_ext(api.h, (P * 3)(*[api.ptr(t) for t in terms]),
                                                     (P * 3)(*[api.ptr(p) for p in d_pts]), 3, api.ptr(acc), G * H,
                                                     L, 0, None))
    out["mpa"] = api.host(acc).copy()
    # encoding over QlP
    dc = api.buf(coeffs.view(np.uint64))
    le = api.empty((2, LP, N))
    api.ok(api.lib.shm_lift_signed_ext(api.h, api.ptr(dc), api.ptr(le), 2, L, None))
    api.ok(api.lib.shm_ntt_forward_ext(api.h, api.ptr(le), 2, L, None))
    out["encode_ext"] = api.host(le).copy()
    lq = api.empty((2, L, N))
    api.ok(api.lib.shm_lift_signed(api.h, api.ptr(dc), api.ptr(lq), 2, L, None))
    api.ok(api.lib.shm_ntt_forward(api.h, api.ptr(lq), 2, L, None))
    out["encode_q"] = api.host(lq).copy()
    out["inputs"] = (sh, ext_in)
    out["elts"], out["keys"] = elts, keys
    return out


def _moddown(api, x, L):
    G, H = x.shape[0], x.shape[1]
    d = api.buf(x)
    o = api.empty((G, H, L, x.shape[-1]))
    api.ok(api.lib.shm_moddown_ext(api.h, api.ptr(d), api.ptr(o), G * H, L, None, 0, None))
    return api.host(o).copy()


@pytest.mark.parametrize("G,n_mem,L", [(2, 3, 3), (1, 2, 6)])
def test_oracle_double_hoisting_identities(G, n_mem, L):
    o = O.Oracle.from_bits(LOG_N, BITS, NP)
    qp = [int(p) for p in o.primes]
    api = Api(ctypes.CDLL(ORACLE_CAPI), qp, device=False)
    r = _ops(api, qp, np.random.default_rng(7 + L), G, n_mem, L)
    sh, _ = r["inputs"]
    assert np.array_equal(_moddown(api, r["extend"], L), sh), "ModDown(P x) = x"
    for e in range(2):
        assert np.array_equal(_moddown(api, r["rot_q"][e], L), r["rot_plain"][e]), "ModDown(Sh-Rot ext) = Sh-Rot"
    # an extended input that is exactly P * sh rotates to the same thing
    N, H = 1 << LOG_N, n_mem + 1
    outs = [api.empty((G, H, L + NP, N)) for _ in range(2)]
    ext = api.buf(r["extend"])
    keys = [api.buf(k) for k in r["keys"]]
    api.ok(api.lib.shm_shared_rotate_ext(api.h, api.ptr(ext), 1, G, n_mem, 2, (U32 * 2)(*r["elts"]),
                                         (P * 2)(*[api.ptr(k) for k in keys]), (P * 2)(*[api.ptr(x) for x in outs]),
                                         L, None, 0, None))
    for e in range(2):
        assert np.array_equal(_moddown(api, outs[e], L), r["rot_plain"][e]), "extended input P x"
    assert np.array_equal(r["encode_ext"][:, :L], r["encode_q"]), "Q limbs of the extended encoding"
    api.close()


@pytest.mark.gpu
@pytest.mark.parametrize("G,n_mem,L", [(2, 3, 3), (1, 2, 6)])
def test_cuda_ext_basis_matches_oracle(G, n_mem, L):
    import shmoai_b200

    o = O.Oracle.from_bits(LOG_N, BITS, NP)
    qp = [int(p) for p in o.primes]
    cu = Api(shmoai_b200.lib(), qp, device=True)
    orc = Api(ctypes.CDLL(ORACLE_CAPI), qp, device=False)
    a = _ops(cu, qp, np.random.default_rng(11 + L), G, n_mem, L)
    b = _ops(orc, qp, np.random.default_rng(11 + L), G, n_mem, L)
    for k in ("extend", "add", "moddown", "mpa", "encode_ext", "encode_q"):
        assert np.array_equal(a[k], b[k]), k
    for k in ("rot_q", "rot_x", "rot_plain"):
        for e in range(2):
            assert np.array_equal(a[k][e], b[k][e]), (k, e)
    cu.close()
    orc.close()
