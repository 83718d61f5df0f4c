"""Device backend of the scale-exact evaluator: every ring operation is one
call into the CUDA library (include/shmoai_ckks.h) on torch device buffers.

Arrays are torch.int64 tensors holding uint64 residues; ciphertext batches are
[n][2][L][N], plaintexts [L][N].  The evaluator (evaluator.py) and the
bootstrapper (bootstrap.py) only talk to this interface, so the same pipeline
code can be checked against another implementation of it.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import check, lib
from .ckks import CKKSContext, _ptr, _stream


class GpuBackend:
    name = "cuda"

    def __init__(self, ctx: CKKSContext, stream: torch.cuda.Stream | None = None):
        self.ctx = ctx
        self.n, self.log_n, self.nq, self.np, self.dnum = ctx.n, ctx.log_n, ctx.nq, ctx.np, ctx.dnum
        self.primes = [int(p) for p in ctx.primes]
        self.stream = stream
        self._ws = None

    # ---------------- memory ----------------
    def workspace(self, words: int) -> torch.Tensor:
        if self._ws is None or self._ws.numel() < words:
            self._ws = torch.empty(int(words), dtype=torch.int64, device=self.ctx.device)
        return self._ws

    def from_host(self, a: np.ndarray) -> torch.Tensor:
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64)).to(self.ctx.device)

    def to_host(self, t: torch.Tensor) -> np.ndarray:
        return t.detach().cpu().numpy().view(np.uint64)

    def empty(self, *shape) -> torch.Tensor:
        return torch.empty(shape, dtype=torch.int64, device=self.ctx.device)

    def stack(self, ts):
        return torch.stack(list(ts))

    def cat(self, ts):
        return torch.cat(list(ts), dim=0)

    def clone(self, t):
        return t.clone()

    def take_poly(self, t, i):
        """Contiguous [n][L][N] copy of polynomial i of every ciphertext in a [n][2][L][N] batch."""
        return t[:, i].contiguous()

    def uniform(self, shape, L_rows, gen: torch.Generator):
        """Uniform residues; the second-to-last axis indexes primes L_rows[...]."""
        pr = torch.tensor([self.primes[i] for i in L_rows], dtype=torch.int64, device=self.ctx.device)
        x = torch.randint(0, 2 ** 62, shape, device=self.ctx.device, generator=gen, dtype=torch.int64)
        return torch.remainder(x, pr.view(*([1] * (len(shape) - 2)), -1, 1))

    # ---------------- ring operations ----------------
    def _s(self):
        return _stream(self.stream)

    def ntt_fwd(self, t):
        return self.ctx.ntt_forward_(t, self.stream)

    def ntt_inv(self, t):
        return self.ctx.ntt_inverse_(t, self.stream)

    def add(self, a, b, out=None):
        return self.ctx.add(a, b, out=out, stream=self.stream)

    def sub(self, a, b, out=None):
        return self.ctx.sub(a, b, out=out, stream=self.stream)

    def neg(self, a, out=None):
        return self.ctx.negate(a, out=out, stream=self.stream)

    def mul_plain(self, ct, pt, out=None):
        return self.ctx.multiply_plain(ct, pt, out=out, stream=self.stream)

    def tensor(self, a, b):
        return self.ctx.multiply(a, b, stream=self.stream)

    def relin(self, ct3, key):
        L = ct3.shape[-2]
        ws = self.workspace(self.ctx.workspace_bytes("keyswitch", ct3.numel() // (3 * L * self.n), L) // 8)
        return self.ctx.relinearize(ct3, key, workspace=ws, stream=self.stream)

    def rescale(self, t):
        p, L = self.ctx._levels(t)
        ws = self.workspace(self.ctx.workspace_bytes("rescale", p, L) // 8)
        return self.ctx.rescale(t, workspace=ws, stream=self.stream)

    def apply_galois(self, ct, elt, key):
        L = ct.shape[-2]
        n_cts = ct.numel() // (2 * L * self.n)
        words = self.ctx.workspace_bytes("keyswitch", n_cts, L) // 8 + n_cts * 2 * L * self.n
        ws = self.workspace(words)
        return self.ctx.apply_galois(ct, elt, key, workspace=ws, stream=self.stream)

    def apply_galois_many(self, ct, elts, keys):
        """Hoisted: one ModUp, one output batch per Galois element."""
        L = ct.shape[-2]
        n_cts = ct.numel() // (2 * L * self.n)
        outs = [torch.empty_like(ct) for _ in elts]
        ws = self.workspace(lib().shm_apply_galois_hoisted_workspace_bytes(self.ctx._h, n_cts, L) // 8)
        k = len(elts)
        E = (ctypes.c_uint32 * k)(*elts)
        K = (ctypes.c_void_p * k)(*[_ptr(x).value for x in keys])
        O = (ctypes.c_void_p * k)(*[_ptr(x).value for x in outs])
        check(lib().shm_apply_galois_hoisted(self.ctx._h, _ptr(ct), k, E, K, O, n_cts, L, _ptr(ws), ws.numel() * 8,
                                             self._s()))
        return outs

    # ---- shared-a groups [G][n + 1][L][N] = (b_0 .. b_{n-1}, a)
    def sh_rotate_many(self, sh, elts, keys):
        """Sh-Rot of every group, one ModUp of each a serving all elements."""
        G, H, L = sh.shape[0], sh.shape[1], sh.shape[2]
        outs = [torch.empty_like(sh) for _ in elts]
        ws = self.workspace(lib().shm_shared_rotate_workspace_bytes(self.ctx._h, G, H - 1, L) // 8)
        k = len(elts)
        E = (ctypes.c_uint32 * k)(*elts)
        K = (ctypes.c_void_p * k)(*[_ptr(x).value for x in keys])
        O = (ctypes.c_void_p * k)(*[_ptr(x).value for x in outs])
        check(lib().shm_shared_rotate_hoisted(self.ctx._h, _ptr(sh), G, H - 1, k, E, K, O, L, _ptr(ws),
                                              ws.numel() * 8, self._s()))
        return outs

    def fmt_forward(self, cts, n, key):
        """[G * n][2][L][N] ciphertexts under s -> [G][n + 1][L][N] shared-a groups."""
        m, L = cts.shape[0], cts.shape[2]
        G = m // n
        out = torch.empty((G, n + 1, L, self.n), dtype=cts.dtype, device=cts.device)
        ws = self.workspace(lib().shm_fmt_switch_forward_workspace_bytes(self.ctx._h, G, n, L) // 8)
        check(lib().shm_fmt_switch_forward(self.ctx._h, _ptr(cts), G, n, _ptr(key), _ptr(out), L, _ptr(ws),
                                           ws.numel() * 8, self._s()))
        return out

    def fmt_backward(self, sh, keys):
        """[G][n + 1][L][N] shared-a groups -> [G * n][2][L][N] ciphertexts under s."""
        G, H, L = sh.shape[0], sh.shape[1], sh.shape[2]
        n = H - 1
        out = torch.empty((G * n, 2, L, self.n), dtype=sh.dtype, device=sh.device)
        ws = self.workspace(lib().shm_fmt_switch_backward_workspace_bytes(self.ctx._h, G, n, L) // 8)
        K = (ctypes.c_void_p * n)(*[_ptr(x).value for x in keys])
        check(lib().shm_fmt_switch_backward(self.ctx._h, _ptr(sh), G, n, K, _ptr(out), L, _ptr(ws), ws.numel() * 8,
                                            self._s()))
        return out

    def permute_plain(self, pt, elt):
        """NTT-domain automorphism of plaintext rows without key switching (key generation only)."""
        return pt[..., self._perm(elt)].contiguous()

    def _perm(self, elt):
        if not hasattr(self, "_perms"):
            self._perms = {}
        if elt not in self._perms:
            log_n, n = self.log_n, self.n
            k = np.arange(n, dtype=np.uint64)
            br = _bitrev(k, log_n)
            e = ((2 * br + 1) * np.uint64(elt)) & np.uint64(2 * n - 1)
            self._perms[elt] = torch.from_numpy(_bitrev((e - 1) >> np.uint64(1), log_n).astype(np.int64)).to(
                self.ctx.device)
        return self._perms[elt]

    def mul_scalar(self, a, residues, out=None):
        p, L = self.ctx._levels(a)
        out = torch.empty_like(a) if out is None else out
        r = np.ascontiguousarray(residues[:L], dtype=np.uint64)
        check(lib().shm_multiply_scalar(self.ctx._h, _ptr(a), r.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                        _ptr(out), p, L, self._s()))
        return out

    def add_scalar(self, ct, residues, out=None):
        p, L = self.ctx._levels(ct)
        out = torch.empty_like(ct) if out is None else out
        r = np.ascontiguousarray(residues[:L], dtype=np.uint64)
        check(lib().shm_add_scalar(self.ctx._h, _ptr(ct), r.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                   _ptr(out), p // 2, L, self._s()))
        return out

    def mul_plain_acc(self, cts, pts, out=None, accumulate=False):
        p, L = self.ctx._levels(cts[0])
        out = torch.empty_like(cts[0]) if out is None else out
        k = len(cts)
        X = (ctypes.c_void_p * k)(*[t.data_ptr() for t in cts])
        P = (ctypes.c_void_p * k)(*[t.data_ptr() for t in pts])
        for t in list(cts) + list(pts):
            _ptr(t)
        check(lib().shm_multiply_plain_accumulate(self.ctx._h, X, P, k, _ptr(out), p, L, 1 if accumulate else 0,
                                                  self._s()))
        return out

    def modraise(self, ct1, L):
        """[n][2][1][N] mod q0 -> [n][2][L][N]"""
        p = ct1.numel() // self.n
        out = self.empty(*(ct1.shape[:-2] + (L, self.n)))
        ws = self.workspace(lib().shm_modraise_workspace_bytes(self.ctx._h, p) // 8)
        check(lib().shm_modraise(self.ctx._h, _ptr(ct1), _ptr(out), p, L, _ptr(ws), ws.numel() * 8, self._s()))
        return out

    def drop(self, t, L_out):
        L = t.shape[-2]
        if L_out == L:
            return t
        p = t.numel() // (L * self.n)
        out = self.empty(*(t.shape[:-2] + (L_out, self.n)))
        check(lib().shm_drop_limbs(self.ctx._h, _ptr(t), _ptr(out), p, L, L_out, self._s()))
        return out

    def synchronize(self):
        torch.cuda.synchronize(self.ctx.device)


def _bitrev(x: np.ndarray, bits: int) -> np.ndarray:
    x = x.astype(np.uint64)
    r = np.zeros_like(x)
    for _ in range(bits):
        r = (r << np.uint64(1)) | (x & np.uint64(1))
        x = x >> np.uint64(1)
    return r
