"""Python binding of the C ABI (include/shmoai_ckks.h) on torch device tensors.

``CKKSContext`` owns a device context (prime chain, twiddles, RNS constants) and
exposes the batched primitives -- NTT, element-wise ops, rescale, key switching,
hoisted and shared-a (Sh-Rot, FmtSwitch) automorphisms, the ct-pt matmul -- for
the parity tests and the kernel benchmarks.  The evaluator, key material and
bootstrapping API (moai::Evaluator and BatchBootstrapper names) is the C++ host
library, bound in shmoai_b200.host.

Tensors are torch.int64 on the context's device holding uint64 residues
(bit pattern preserved), shaped [..., L, N].  Errors raise ShmError with the
library's message (the reference throws std::invalid_argument).
"""
from __future__ import annotations

import ctypes

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


class Graph:
    """A recorded sequence of library calls (shm_graph); launch() replays it with one launch."""

    def __init__(self, ctx: "CKKSContext", handle, stream):
        self._ctx, self._g, self._s = ctx, handle, stream

    @property
    def kernels(self) -> int:
        return int(lib().shm_graph_kernels(self._g))

    def launch(self, stream=None):
        check(lib().shm_graph_launch(self._g, _stream(stream)))

    def close(self):
        if getattr(self, "_g", None):
            lib().shm_graph_destroy(self._g)
            lib().shm_stream_destroy(self._ctx._h, self._s)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


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

    def capture(self, fn) -> "Graph":
        """A CUDA graph (shm_graph_begin / shm_graph_end) of the library calls fn() makes.
        fn runs twice on a private stream, once as is and once under capture; it must
        allocate nothing (pass `out` and `workspace` tensors) and only touch tensors that
        outlive the graph.  Graph.launch() replays it on the current stream."""
        s = ctypes.c_void_p()
        check(lib().shm_stream_create(self._h, ctypes.byref(s)))
        ext = torch.cuda.ExternalStream(s.value, device=self.device)
        torch.cuda.synchronize(self.device)  # inputs made on other streams are complete
        g = ctypes.c_void_p()
        try:
            with torch.cuda.stream(ext):
                fn()
                check(lib().shm_graph_begin(self._h, s))
                try:
                    fn()
                finally:
                    rc = lib().shm_graph_end(self._h, s, ctypes.byref(g))
                check(rc)
        except BaseException:
            if g.value:
                lib().shm_graph_destroy(g)
            lib().shm_stream_destroy(self._h, s)
            raise
        return Graph(self, g, s)

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

    def multiply(self, a, b, out=None, stream=None):
        """[n][2][L][N] x [n][2][L][N] -> [n][3][L][N] (a single ct may omit the batch axis)."""
        p, L = self._levels(a)
        n_cts = p // 2
        out = self.empty(*(a.shape[:-3] + (3, L, self.n))) if out is None else out
        check(lib().shm_multiply(self._h, _ptr(a), _ptr(b), _ptr(out), n_cts, L, _stream(stream)))
        return out

    def rescale(self, a, out=None, workspace=None, stream=None):
        p, L = self._levels(a)
        out = self.empty(*(a.shape[:-2] + (L - 1, self.n))) if out is None else out
        ws, wsb = self._ws(workspace)
        check(lib().shm_rescale(self._h, _ptr(a), _ptr(out), p, L, ws, wsb, _stream(stream)))
        return out

    def modraise(self, a, L: int, workspace=None, stream=None):
        """[..][1][N] one-limb polynomials (mod q0, NTT form) -> [..][L][N] by the centred lift."""
        p = a.numel() // self.n
        out = self.empty(*(a.shape[:-2] + (L, self.n)))
        ws, wsb = self._ws(workspace)
        check(lib().shm_modraise(self._h, _ptr(a), _ptr(out), p, L, ws, wsb, _stream(stream)))
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

    # ---------------- hoisted and shared-a automorphisms ----------------
    def apply_galois_hoisted(self, ct, elts, keys, stream=None):
        """[n][2][L][N]: one ModUp of the c1 polynomials, one output batch per Galois element."""
        p, L = self._levels(ct)
        outs = [torch.empty_like(ct) for _ in elts]
        ws = self.empty(max(1, lib().shm_apply_galois_hoisted_workspace_bytes(self._h, p // 2, L) // 8))
        k = len(elts)
        E = (ctypes.c_uint32 * k)(*elts)
        K = (ctypes.c_void_p * k)(*[_ptr(x).value for x in keys])
        O = (ctypes.c_void_p * k)(*[_ptr(x).value for x in outs])
        check(lib().shm_apply_galois_hoisted(self._h, _ptr(ct), k, E, K, O, p // 2, L, _ptr(ws), ws.numel() * 8,
                                             _stream(stream)))
        return outs

    def shared_rotate_hoisted(self, sh, elts, keys, stream=None):
        """Shared-a groups [G][n + 1][L][N]: Sh-Rot by every element, one ModUp of each a."""
        G, H, L = sh.shape[0], sh.shape[1], sh.shape[2]
        outs = [torch.empty_like(sh) for _ in elts]
        ws = self.empty(max(1, lib().shm_shared_rotate_workspace_bytes(self._h, G, H - 1, L) // 8))
        k = len(elts)
        E = (ctypes.c_uint32 * k)(*elts)
        K = (ctypes.c_void_p * k)(*[_ptr(x).value for x in keys])
        O = (ctypes.c_void_p * k)(*[_ptr(x).value for x in outs])
        check(lib().shm_shared_rotate_hoisted(self._h, _ptr(sh), G, H - 1, k, E, K, O, L, _ptr(ws), ws.numel() * 8,
                                              _stream(stream)))
        return outs

    def shared_rotate(self, sh, elt: int, key, stream=None):
        """Shared-a groups [G][n + 1][L][N]: Sh-Rot by one element in the reference's order
        (automorphism, then ModUp of a; ShRotate.cu:201-257)."""
        G, H, L = sh.shape[0], sh.shape[1], sh.shape[2]
        out = torch.empty_like(sh)
        ws = self.empty(max(1, lib().shm_shared_rotate_one_workspace_bytes(self._h, G, H - 1, L) // 8))
        check(lib().shm_shared_rotate(self._h, _ptr(sh), G, H - 1, elt, _ptr(key), _ptr(out), L, _ptr(ws),
                                      ws.numel() * 8, _stream(stream)))
        return out

    def fmt_forward(self, cts, n, key, stream=None):
        """[G * n][2][L][N] ciphertexts under s -> [G][n + 1][L][N] shared-a groups."""
        m, L = cts.shape[0], cts.shape[2]
        G = m // n
        out = self.empty(G, n + 1, L, self.n)
        ws = self.empty(max(1, lib().shm_fmt_switch_forward_workspace_bytes(self._h, G, n, L) // 8))
        check(lib().shm_fmt_switch_forward(self._h, _ptr(cts), G, n, _ptr(key), _ptr(out), L, _ptr(ws),
                                           ws.numel() * 8, _stream(stream)))
        return out

    def fmt_backward(self, sh, keys, stream=None):
        """[G][n + 1][L][N] shared-a groups -> [G * n][2][L][N] ciphertexts under s."""
        G, H, L = sh.shape[0], sh.shape[1], sh.shape[2]
        n = H - 1
        out = self.empty(G * n, 2, L, self.n)
        ws = self.empty(max(1, lib().shm_fmt_switch_backward_workspace_bytes(self._h, G, n, L) // 8))
        K = (ctypes.c_void_p * n)(*[_ptr(x).value for x in keys])
        check(lib().shm_fmt_switch_backward(self._h, _ptr(sh), G, n, K, _ptr(out), L, _ptr(ws), ws.numel() * 8,
                                            _stream(stream)))
        return out
