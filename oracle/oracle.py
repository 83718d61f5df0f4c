"""ctypes face of the CPU oracle (oracle/ckks_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline leg as the checker.  The product package
(``shmoai_b200``) never imports it.

Besides the oracle arithmetic this module holds the deterministic counter
generator that the golden harness (oracle/ref_golden.cu) uses for inputs and
key material, so a test can rebuild any golden input bit for bit.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libckks_oracle.so")
REF_HOST_PATH = os.path.join(HERE, "_ref", "libref_host.so")

# Parameter sets of the golden harness (name -> (log_n, bit sizes, special count)).
PARAM_SETS = {
    "tiny": (12, [60] + [50] * 5 + [60] * 2, 2),
    "prim": (16, [60] + [50] * 23 + [60] * 8, 8),
    "boot": (16, [51] + [46] * 20 + [51] * 14 + [51] * 5, 5),
}

_u64p = ctypes.POINTER(ctypes.c_uint64)
_lib = None


def build():
    """Compile the oracle library (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        u32, u64 = ctypes.c_uint32, ctypes.c_uint64
        L.orc_gen_primes.argtypes = [u32, ctypes.POINTER(ctypes.c_int), u32, _u64p]
        L.orc_minimal_root.argtypes = [u64, u32]
        L.orc_minimal_root.restype = u64
        L.orc_invmod.argtypes = [u64, u64]
        L.orc_invmod.restype = u64
        L.orc_ntt_tables.argtypes = [u64, u32, _u64p, _u64p]
        L.orc_ctx_create.argtypes = [u32, _u64p, u32, u32]
        L.orc_ctx_create.restype = vp
        L.orc_ctx_destroy.argtypes = [vp]
        L.orc_ntt.argtypes = [vp, _u64p, u32, u32, ctypes.c_int]
        L.orc_add.argtypes = [vp, _u64p, _u64p, _u64p, u32, u32]
        L.orc_multiply_plain.argtypes = [vp, _u64p, _u64p, _u64p, u32, u32]
        L.orc_tensor.argtypes = [vp, _u64p, _u64p, _u64p, u32]
        L.orc_rescale.argtypes = [vp, _u64p, _u64p, u32, u32]
        L.orc_galois_perm.argtypes = [u32, u32, ctypes.POINTER(ctypes.c_uint32)]
        L.orc_apply_galois.argtypes = [vp, _u64p, _u64p, u32, u32, u32]
        L.orc_galois_elt_from_step.argtypes = [u32, ctypes.c_int]
        L.orc_galois_elt_from_step.restype = u32
        L.orc_modup.argtypes = [vp, _u64p, u32, _u64p]
        L.orc_keyswitch.argtypes = [vp, _u64p, u32, _u64p, u32, _u64p]
        L.orc_relinearize.argtypes = [vp, _u64p, u32, _u64p, u32, _u64p]
        L.orc_apply_galois_ct.argtypes = [vp, _u64p, u32, u32, _u64p, u32, _u64p]
        L.orc_ctpt_matmul.argtypes = [vp, _u64p, ctypes.POINTER(ctypes.c_int64), u32, u32, u32, _u64p]
        L.orc_apply_galois_hoisted.argtypes = [vp, _u64p, u32, u32, ctypes.POINTER(ctypes.c_uint32),
                                               ctypes.POINTER(_u64p), u32, ctypes.POINTER(_u64p)]
        L.orc_shared_rotate_hoisted.argtypes = [vp, _u64p, u32, u32, u32, ctypes.POINTER(ctypes.c_uint32),
                                                ctypes.POINTER(_u64p), ctypes.POINTER(_u64p)]
        L.orc_fmt_forward.argtypes = [vp, _u64p, u32, u32, _u64p, _u64p]
        L.orc_exact_extend.argtypes = [vp, _u64p, u32, u32, _u64p]
        L.orc_modraise.argtypes = [vp, _u64p, _u64p, u32, u32]
        L.orc_fmt_backward.argtypes = [vp, _u64p, u32, u32, ctypes.POINTER(_u64p), _u64p]
        L.orc_signed_residue.argtypes = [ctypes.c_int64, u64]
        L.orc_signed_residue.restype = u64
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u64p)


def gen_primes(log_n: int, bits) -> np.ndarray:
    out = np.zeros(len(bits), dtype=np.uint64)
    arr = (ctypes.c_int * len(bits))(*bits)
    if lib().orc_gen_primes(log_n, arr, len(bits), _p(out)) != 0:
        raise ValueError("not enough primes")
    return out


def ntt_tables(q: int, log_n: int):
    n = 1 << log_n
    rp = np.zeros(n, dtype=np.uint64)
    irp = np.zeros(n, dtype=np.uint64)
    lib().orc_ntt_tables(q, log_n, _p(rp), _p(irp))
    return rp, irp


def galois_perm(log_n: int, elt: int) -> np.ndarray:
    out = np.zeros(1 << log_n, dtype=np.uint32)
    lib().orc_galois_perm(log_n, elt, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    return out


def galois_elt_from_step(log_n: int, step: int) -> int:
    return int(lib().orc_galois_elt_from_step(log_n, step))


class Oracle:
    """Oracle context over a prime chain Q (nq primes) followed by P (np)."""

    def __init__(self, log_n: int, primes, nq: int, np_: int):
        self.log_n, self.n, self.nq, self.np = log_n, 1 << log_n, nq, np_
        self.primes = np.ascontiguousarray(primes, dtype=np.uint64)
        self.dnum = nq // np_ if np_ else 0
        self._h = lib().orc_ctx_create(log_n, _p(self.primes), nq, np_)

    @classmethod
    def from_bits(cls, log_n: int, bits, np_: int) -> "Oracle":
        return cls(log_n, gen_primes(log_n, bits), len(bits) - np_, np_)

    @classmethod
    def param_set(cls, name: str) -> "Oracle":
        log_n, bits, np_ = PARAM_SETS[name]
        return cls.from_bits(log_n, bits, np_)

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _lib is not None:
            _lib.orc_ctx_destroy(h)

    # --- arithmetic (all arrays uint64, C-contiguous, limbs under primes[0..L)) ---
    def ntt(self, a: np.ndarray, inverse=False) -> np.ndarray:
        a = np.array(a, dtype=np.uint64, copy=True, order="C")
        L = a.shape[-2]
        lib().orc_ntt(self._h, _p(a), a.size // (L * self.n), L, 1 if inverse else 0)
        return a

    def intt(self, a):
        return self.ntt(a, inverse=True)

    def add(self, a, b):
        out = np.empty_like(a)
        L = a.shape[-2]
        lib().orc_add(self._h, _p(a), _p(b), _p(out), a.size // (L * self.n), L)
        return out

    def multiply_plain(self, ct, pt):
        out = np.empty_like(ct)
        L = ct.shape[-2]
        lib().orc_multiply_plain(self._h, _p(ct), _p(pt), _p(out), ct.size // (L * self.n), L)
        return out

    def tensor(self, a, b):
        L = a.shape[-2]
        out = np.empty((3, L, self.n), dtype=np.uint64)
        lib().orc_tensor(self._h, _p(a), _p(b), _p(out), L)
        return out

    def rescale(self, a):
        L = a.shape[-2]
        npoly = a.size // (L * self.n)
        out = np.empty(a.shape[:-2] + (L - 1, self.n), dtype=np.uint64)
        lib().orc_rescale(self._h, _p(a), _p(out), npoly, L)
        return out

    def apply_galois(self, a, elt):
        L = a.shape[-2]
        out = np.empty_like(a)
        lib().orc_apply_galois(self._h, _p(a), _p(out), a.size // (L * self.n), L, elt)
        return out

    def modup(self, d):
        L = d.shape[-2]
        beta = -(-L // self.np)
        out = np.empty((beta, L + self.np, self.n), dtype=np.uint64)
        lib().orc_modup(self._h, _p(d), L, _p(out))
        return out

    def keyswitch(self, d, key):
        L = d.shape[-2]
        out = np.empty((2, L, self.n), dtype=np.uint64)
        lib().orc_keyswitch(self._h, _p(d), L, _p(key), self.dnum, _p(out))
        return out

    def relinearize(self, ct3, key):
        L = ct3.shape[-2]
        out = np.empty((2, L, self.n), dtype=np.uint64)
        lib().orc_relinearize(self._h, _p(ct3), L, _p(key), self.dnum, _p(out))
        return out

    def apply_galois_ct(self, ct, elt, key):
        L = ct.shape[-2]
        out = np.empty((2, L, self.n), dtype=np.uint64)
        lib().orc_apply_galois_ct(self._h, _p(ct), L, elt, _p(key), self.dnum, _p(out))
        return out

    def apply_galois_hoisted(self, ct, elts, keys):
        """[2][L][N] ciphertext, one ModUp, one output per Galois element."""
        L = ct.shape[-2]
        ct = np.ascontiguousarray(ct, dtype=np.uint64)
        keys = [np.ascontiguousarray(k, dtype=np.uint64) for k in keys]
        outs = [np.empty((2, L, self.n), dtype=np.uint64) for _ in elts]
        e = (ctypes.c_uint32 * len(elts))(*elts)
        kp = (_u64p * len(keys))(*[_p(k) for k in keys])
        op = (_u64p * len(outs))(*[_p(o) for o in outs])
        lib().orc_apply_galois_hoisted(self._h, _p(ct), L, len(elts), e, kp, self.dnum, op)
        return outs

    # ---- shared-a groups [n + 1][L][N] = (b_0 .. b_{n-1}, a)
    def shared_rotate_hoisted(self, sh, elts, keys):
        """One ModUp of a; per element a rotated group with keys[e] [dnum][n+1][QP][N]."""
        H, L = sh.shape[0], sh.shape[1]
        sh = np.ascontiguousarray(sh, dtype=np.uint64)
        keys = [np.ascontiguousarray(k, dtype=np.uint64) for k in keys]
        outs = [np.empty((H, L, self.n), dtype=np.uint64) for _ in elts]
        e = (ctypes.c_uint32 * len(elts))(*elts)
        kp = (_u64p * len(keys))(*[_p(k) for k in keys])
        op = (_u64p * len(outs))(*[_p(o) for o in outs])
        lib().orc_shared_rotate_hoisted(self._h, _p(sh), H - 1, L, len(elts), e, kp, op)
        return outs

    def modraise(self, a, L: int):
        """[..][1][N] polynomials mod q0 (NTT form) -> [..][L][N] by the centred lift."""
        a = np.ascontiguousarray(a, dtype=np.uint64)
        m = a.size // self.n
        out = np.empty(a.shape[:-2] + (L, self.n), dtype=np.uint64)
        lib().orc_modraise(self._h, _p(a), _p(out), m, L)
        return out

    def exact_extend(self, a):
        """[..][L][N] NTT-form polynomials -> [..][L + np][N]: the Ql rows copied, the P rows
        the floor-corrected CRT extension of FmtSwitch.cu:86-106 (NTT form)."""
        L = a.shape[-2]
        a = np.ascontiguousarray(a, dtype=np.uint64)
        m = int(np.prod(a.shape[:-2], dtype=np.int64))
        out = np.empty(a.shape[:-2] + (L + self.np, self.n), dtype=np.uint64)
        lib().orc_exact_extend(self._h, _p(a), m, L, _p(out))
        return out

    def shared_rotate(self, sh, elt, key):
        """Sh-Rot of one group [n+1][L][N] in the reference's order (ShRotate.cu:218-256): the automorphism on
        every row first, then one ModUp of the rotated a and the key switch."""
        return self.shared_rotate_hoisted(self.apply_galois(sh, elt), [1], [key])[0]

    def fmt_forward(self, cts, key):
        """[n][2][L][N] ciphertexts under s -> one shared-a group [n+1][L][N]."""
        m, _, L, _ = cts.shape
        cts = np.ascontiguousarray(cts, dtype=np.uint64)
        key = np.ascontiguousarray(key, dtype=np.uint64)
        out = np.empty((m + 1, L, self.n), dtype=np.uint64)
        lib().orc_fmt_forward(self._h, _p(cts), m, L, _p(key), _p(out))
        return out

    def fmt_backward(self, sh, keys):
        """shared-a group [n+1][L][N] -> [n][2][L][N] under s; keys[i] [dnum][2][QP][N]."""
        H, L = sh.shape[0], sh.shape[1]
        sh = np.ascontiguousarray(sh, dtype=np.uint64)
        keys = [np.ascontiguousarray(k, dtype=np.uint64) for k in keys]
        out = np.empty((H - 1, 2, L, self.n), dtype=np.uint64)
        kp = (_u64p * len(keys))(*[_p(k) for k in keys])
        lib().orc_fmt_backward(self._h, _p(sh), H - 1, L, kp, _p(out))
        return out

    def ctpt_matmul(self, X, W):
        n_in, _, L, _ = X.shape
        n_out = W.shape[1]
        W = np.ascontiguousarray(W, dtype=np.int64)
        Y = np.empty((n_out, 2, L, self.n), dtype=np.uint64)
        lib().orc_ctpt_matmul(self._h, _p(X), W.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), n_in, n_out, L,
                              _p(Y))
        return Y


# ---------------------------------------------------------------------------
# Deterministic counter generator shared with oracle/ref_golden.cu

_GOLD = np.uint64(0x9E3779B97F4A7C15)


def sm64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = np.asarray(x, dtype=np.uint64) + _GOLD
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def fill(tag: int, shape, row_moduli) -> np.ndarray:
    """Array of `shape` whose flat element e is sm64((tag << 40) + e) mod the
    modulus of its row (rows are the last axis)."""
    total = int(np.prod(shape))
    n = shape[-1]
    e = np.arange(total, dtype=np.uint64)
    v = sm64(np.uint64(tag << 40) + e)
    mods = np.repeat(np.asarray(row_moduli, dtype=np.uint64), n)
    return (v % mods).reshape(shape)


def checksum(a: np.ndarray) -> str:
    a = np.ascontiguousarray(a, dtype=np.uint64).ravel()
    with np.errstate(over="ignore"):
        e = np.arange(a.size, dtype=np.uint64) * _GOLD
        h = sm64(a ^ e).sum(dtype=np.uint64)
    return "%016x" % int(h)


def weight(tag: int, i) -> np.ndarray:
    """N(0,.)-free reproducible weights in [-0.08, 0.08): a 53-bit integer times a constant."""
    i = np.asarray(i, dtype=np.uint64)
    m = (sm64(np.uint64(tag << 40) + i) >> np.uint64(11)).astype(np.int64) - (1 << 52)
    return m.astype(np.float64) * (0.08 / 4503599627370496.0)


def ref_host():
    """The reference's own host number theory (oracle/_ref/libref_host.so), or None if not built."""
    if not os.path.exists(REF_HOST_PATH):
        return None
    L = ctypes.CDLL(REF_HOST_PATH)
    L.ref_create_primes.argtypes = [ctypes.c_uint32, ctypes.POINTER(ctypes.c_int), ctypes.c_uint32, _u64p]
    L.ref_ntt_tables.argtypes = [ctypes.c_uint32, ctypes.c_uint64, _u64p, _u64p, _u64p, _u64p]
    L.ref_base_converter.argtypes = [_u64p, ctypes.c_uint32, _u64p, ctypes.c_uint32, _u64p, _u64p]
    return L
