"""Host-side mirror of ShMOAI's evaluator interface over the C ABI.

``CKKSContext`` owns a device context (prime chain, twiddles, RNS constants)
and exposes the batched entry points of include/shmoai_ckks.h on torch
device tensors.  ``Ciphertext`` / ``Plaintext`` / ``Evaluator`` mirror the
names, argument meaning and error behaviour of ``moai::Evaluator``
(src/include/source/ckks_evaluator_parallel.cuh:150-562): level or scale
mismatches raise ``ValueError`` (the reference throws std::invalid_argument).

Tensors are torch.int64 on the context's device holding uint64 residues
(bit pattern preserved), shaped [..., L, N].
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from ._lib import check, lib


def _ptr(t: torch.Tensor | None):
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous() or t.dtype != torch.int64:
        raise ValueError("expected a contiguous int64 CUDA tensor")
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def to_device(a: np.ndarray, device="cuda") -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64)).to(device)


def to_host(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().numpy().view(np.uint64)


class CKKSContext:
    """Device context over Q (n_q primes) followed by special primes P (n_p)."""

    def __init__(self, log_n: int, bits=None, n_special: int = 0, primes=None, device: int = 0):
        h = ctypes.c_void_p()
        if primes is not None:
            pr = np.ascontiguousarray(primes, dtype=np.uint64)
            nq = len(pr) - n_special
            check(lib().shm_context_create_from_primes(ctypes.byref(h), log_n,
                                                       pr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), nq,
                                                       n_special, device))
        else:
            arr = (ctypes.c_int * len(bits))(*bits)
            check(lib().shm_context_create(ctypes.byref(h), log_n, arr, len(bits) - n_special, n_special, device))
        self._h = h
        self.device = torch.device("cuda", device)
        v = [ctypes.c_uint32() for _ in range(4)]
        check(lib().shm_context_info(h, *[ctypes.byref(x) for x in v]))
        self.log_n, self.nq, self.np, self.dnum = (x.value for x in v)
        self.n = 1 << self.log_n
        pr = np.zeros(self.nq + self.np, dtype=np.uint64)
        check(lib().shm_context_primes(h, pr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        self.primes = pr

    def close(self):
        if getattr(self, "_h", None):
            lib().shm_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------- helpers ----------------
    def empty(self, *shape) -> torch.Tensor:
        return torch.empty(shape, dtype=torch.int64, device=self.device)

    def _levels(self, t: torch.Tensor) -> tuple[int, int]:
        """(number of polynomials, L) of a [..., L, N] tensor."""
        if t.shape[-1] != self.n:
            raise ValueError("last axis must be N")
        L = t.shape[-2]
        return t.numel() // (L * self.n), L

    # ---------------- primitives ----------------
    def ntt_forward_(self, t, stream=None):
        p, L = self._levels(t)
        check(lib().shm_ntt_forward(self._h, _ptr(t), p, L, _stream(stream)))
        return t

    def ntt_inverse_(self, t, stream=None):
        p, L = self._levels(t)
        check(lib().shm_ntt_inverse(self._h, _ptr(t), p, L, _stream(stream)))
        return t

    def add(self, a, b, out=None, stream=None):
        p, L = self._levels(a)
        out = torch.empty_like(a) if out is None else out
        check(lib().shm_add(self._h, _ptr(a), _ptr(b), _ptr(out), p, L, _stream(stream)))
        return out

    def sub(self, a, b, out=None, stream=None):
        p, L = self._levels(a)
        out = torch.empty_like(a) if out is None else out
        check(lib().shm_sub(self._h, _ptr(a), _ptr(b), _ptr(out), p, L, _stream(stream)))
        return out

    def negate(self, a, out=None, stream=None):
        p, L = self._levels(a)
        out = torch.empty_like(a) if out is None else out
        check(lib().shm_negate(self._h, _ptr(a), _ptr(out), p, L, _stream(stream)))
        return out

    def multiply_plain(self, ct, pt, out=None, stream=None):
        p, L = self._levels(ct)
        out = torch.empty_like(ct) if out is None else out
        check(lib().shm_multiply_plain(self._h, _ptr(ct), _ptr(pt), _ptr(out), p, L, _stream(stream)))
        return out

    def multiply(self, a, b, stream=None):
        """[n][2][L][N] x [n][2][L][N] -> [n][3][L][N] (a single ct may omit the batch axis)."""
        p, L = self._levels(a)
        n_cts = p // 2
        out = self.empty(*(a.shape[:-3] + (3, L, self.n)))
        check(lib().shm_multiply(self._h, _ptr(a), _ptr(b), _ptr(out), n_cts, L, _stream(stream)))
        return out

    def rescale(self, a, out=None, workspace=None, stream=None):
        p, L = self._levels(a)
        out = self.empty(*(a.shape[:-2] + (L - 1, self.n))) if out is None else out
        ws, wsb = self._ws(workspace)
        check(lib().shm_rescale(self._h, _ptr(a), _ptr(out), p, L, ws, wsb, _stream(stream)))
        return out

    def keyswitch(self, d, key, workspace=None, stream=None):
        p, L = self._levels(d)
        out = self.empty(p, 2, L, self.n)
        ws, wsb = self._ws(workspace)
        check(lib().shm_keyswitch(self._h, _ptr(d), _ptr(key), _ptr(out), p, L, ws, wsb, _stream(stream)))
        return out

    def relinearize(self, ct3, key, out=None, workspace=None, stream=None):
        p, L = self._levels(ct3)
        n_cts = p // 3
        out = self.empty(*(ct3.shape[:-3] + (2, L, self.n))) if out is None else out
        ws, wsb = self._ws(workspace)
        check(lib().shm_relinearize(self._h, _ptr(ct3), _ptr(key), _ptr(out), n_cts, L, ws, wsb, _stream(stream)))
        return out

    def galois_elt(self, step: int) -> int:
        e = lib().shm_galois_elt_from_step(self._h, step)
        if e == 0:
            raise ValueError("step count too large")
        return e

    def apply_galois(self, ct, elt: int, key, out=None, workspace=None, stream=None):
        p, L = self._levels(ct)
        out = torch.empty_like(ct) if out is None else out
        ws, wsb = self._ws(workspace)
        check(lib().shm_apply_galois(self._h, _ptr(ct), elt, _ptr(key), _ptr(out), p // 2, L, ws, wsb,
                                     _stream(stream)))
        return out

    def rotate(self, ct, step: int, key, out=None, workspace=None, stream=None):
        return self.apply_galois(ct, self.galois_elt(step), key, out, workspace, stream)

    def ctpt_matmul(self, X, W, out=None, workspace=None, stream=None):
        """X [n_in][2][L][N], W int64 [n_in][n_out] (encoded integer weights) -> Y [n_out][2][L][N]."""
        n_in, L = X.shape[0], X.shape[-2]
        n_out = W.shape[1]
        W = W.contiguous()
        out = self.empty(n_out, 2, L, self.n) if out is None else out
        ws, wsb = self._ws(workspace)
        check(lib().shm_ctpt_matmul(self._h, _ptr(X), _ptr(W), _ptr(out), n_in, n_out, L, ws, wsb,
                                    _stream(stream)))
        return out

    def workspace_bytes(self, op: str, n: int, L: int, n_out: int = 0) -> int:
        f = {"rescale": lib().shm_rescale_workspace_bytes, "keyswitch": lib().shm_keyswitch_workspace_bytes}
        if op == "ctpt":
            return lib().shm_ctpt_matmul_workspace_bytes(self._h, n, n_out, L)
        return f[op](self._h, n, L)

    @staticmethod
    def _ws(workspace):
        if workspace is None:
            return None, 0
        return _ptr(workspace), workspace.numel() * 8


# ---------------------------------------------------------------------------
# moai-style objects


@dataclass
class Ciphertext:
    data: torch.Tensor  # [size][L][N]
    scale: float
    is_ntt_form: bool = True

    @property
    def coeff_modulus_size(self) -> int:
        return self.data.shape[-2]

    @property
    def size(self) -> int:
        return self.data.shape[0]


@dataclass
class Plaintext:
    data: torch.Tensor  # [L][N]
    scale: float


@dataclass
class Evaluator:
    """moai::Evaluator method names over one CKKSContext."""

    ctx: CKKSContext
    relin_key: torch.Tensor | None = None
    galois_keys: dict = field(default_factory=dict)  # elt -> key tensor

    def _same(self, a: Ciphertext, b: Ciphertext, rel=1e-12):
        if a.coeff_modulus_size != b.coeff_modulus_size:
            raise ValueError("encrypted1 and encrypted2 parameter mismatch")
        if abs(a.scale - b.scale) > rel * max(a.scale, b.scale):
            raise ValueError("scale mismatch")

    def add(self, a: Ciphertext, b: Ciphertext) -> Ciphertext:
        self._same(a, b)
        return Ciphertext(self.ctx.add(a.data, b.data), a.scale)

    def add_inplace(self, a: Ciphertext, b: Ciphertext):
        self._same(a, b)
        self.ctx.add(a.data, b.data, out=a.data)

    def sub(self, a: Ciphertext, b: Ciphertext) -> Ciphertext:
        self._same(a, b)
        return Ciphertext(self.ctx.sub(a.data, b.data), a.scale)

    def negate(self, a: Ciphertext) -> Ciphertext:
        return Ciphertext(self.ctx.negate(a.data), a.scale)

    def multiply_plain(self, a: Ciphertext, p: Plaintext) -> Ciphertext:
        if p.data.shape[-2] != a.coeff_modulus_size:
            raise ValueError("encrypted and plain parameter mismatch")
        return Ciphertext(self.ctx.multiply_plain(a.data, p.data), a.scale * p.scale)

    def multiply(self, a: Ciphertext, b: Ciphertext) -> Ciphertext:
        self._same(a, b, rel=float("inf"))
        return Ciphertext(self.ctx.multiply(a.data, b.data), a.scale * b.scale)

    def relinearize_inplace(self, a: Ciphertext):
        if self.relin_key is None:
            raise ValueError("relinearization key not set")
        if a.size != 3:
            raise ValueError("relinearize needs a size-3 ciphertext")
        a.data = self.ctx.relinearize(a.data, self.relin_key)

    def rescale_to_next_inplace(self, a: Ciphertext):
        if a.coeff_modulus_size < 2:
            raise ValueError("end of modulus switching chain reached")
        q_last = float(self.ctx.primes[a.coeff_modulus_size - 1])
        a.data = self.ctx.rescale(a.data)
        a.scale = a.scale / q_last

    def apply_galois_inplace(self, a: Ciphertext, elt: int):
        if elt not in self.galois_keys:
            raise ValueError("Galois elt not present")
        a.data = self.ctx.apply_galois(a.data, elt, self.galois_keys[elt])

    def rotate_vector_inplace(self, a: Ciphertext, step: int):
        self.apply_galois_inplace(a, self.ctx.galois_elt(step))

    def rotate_vector(self, a: Ciphertext, step: int) -> Ciphertext:
        out = Ciphertext(a.data.clone(), a.scale)
        self.rotate_vector_inplace(out, step)
        return out

    def complex_conjugate_inplace(self, a: Ciphertext):
        self.apply_galois_inplace(a, self.ctx.galois_elt(0))

    def transform_from_ntt_inplace(self, a: Ciphertext):
        self.ctx.ntt_inverse_(a.data)
        a.is_ntt_form = False

    def transform_to_ntt_inplace(self, a: Ciphertext):
        self.ctx.ntt_forward_(a.data)
        a.is_ntt_form = True
