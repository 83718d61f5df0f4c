"""Python binding of the C++ host library (include/shmoai_host.h) through ctypes.

`Host` owns a context, the secret key and the evaluation keys; `Ct` owns one
ciphertext batch (ordinary [count][2][L][N], or shared-a groups
[count][members + 1][L][N]); `Bootstrapper` runs S2C-first (shared-a) batched
bootstrapping.  By default the CUDA build (shmoai_b200/_build/libshmoai_host.so) is
loaded; `Host(..., lib=path)` loads another build of the same library.
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

_DIR = os.path.dirname(os.path.abspath(__file__))
PRODUCT_LIB = os.path.join(_DIR, "_build", "libshmoai_host.so")

_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_libs: dict[str, ctypes.CDLL] = {}


def build(jobs: int = 8) -> str:
    """Build the CUDA library and the host library in place; returns the host library path."""
    from ._lib import build as build_all

    build_all(jobs)
    return PRODUCT_LIB


def load(path: str | None = None) -> ctypes.CDLL:
    path = os.path.abspath(path or PRODUCT_LIB)
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise RuntimeError(f"host library not built: {path} (run shmoai_b200.host.build())")
    L = ctypes.CDLL(path)
    u64p, dp, i32 = ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_double), ctypes.c_int
    pp = ctypes.POINTER(_P)
    sig = {
        "shm_host_last_error": (ctypes.c_char_p, []),
        "shm_host_create": (i32, [pp, _U32, u64p, _U32, _U32, i32, _U32, ctypes.c_uint64]),
        "shm_host_create_from_bits": (i32, [pp, _U32, ctypes.POINTER(ctypes.c_int), _U32, _U32, i32, _U32,
                                            ctypes.c_uint64]),
        "shm_host_primes": (i32, [_P, u64p]),
        "shm_host_destroy": (None, [_P]),
        "shm_host_context": (_P, [_P]),
        "shm_host_synchronize": (i32, [_P]),
        "shm_host_device_memory": (i32, [_P, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t),
                                         i32]),
        "shm_host_gen_relin_key": (i32, [_P]),
        "shm_host_gen_galois_keys": (i32, [_P, ctypes.POINTER(_U32), _U32]),
        "shm_host_gen_shared_keys": (i32, [_P, _U32, _U32, ctypes.POINTER(_U32), _U32]),
        "shm_host_galois_elt": (_U32, [_P, i32]),
        "shm_host_encrypt": (i32, [_P, dp, dp, _U32, _U32, _U32, ctypes.c_double, pp]),
        "shm_host_gen_public_key": (i32, [_P, ctypes.c_uint64]),
        "shm_host_encrypt_public": (i32, [_P, dp, dp, _U32, _U32, _U32, ctypes.c_double, pp]),
        "shm_host_batch_input": (i32, [_P, dp, _U32, _U32, _U32, ctypes.c_double, _U32, pp]),
        "shm_host_bias_vec": (i32, [ctypes.POINTER(ctypes.c_int), _U32, _U32, ctypes.POINTER(ctypes.c_int)]),
        "shm_host_decrypt": (i32, [_P, _P, dp, dp]),
        "shm_ct_from_host": (i32, [_P, u64p, _U32, _U32, _U32, ctypes.c_double, i32, pp]),
        "shm_ct_to_host": (i32, [_P, _P, u64p]),
        "shm_ct_info": (i32, [_P, ctypes.POINTER(_U32), ctypes.POINTER(_U32), ctypes.POINTER(_U32), dp,
                              ctypes.POINTER(i32)]),
        "shm_ct_device_data": (_P, [_P]),
        "shm_ct_destroy": (None, [_P]),
        "shm_host_add": (i32, [_P, _P, _P, pp]),
        "shm_host_sub": (i32, [_P, _P, _P, pp]),
        "shm_host_multiply": (i32, [_P, _P, _P, pp]),
        "shm_host_rescale": (i32, [_P, _P, pp]),
        "shm_host_multiply_const": (i32, [_P, _P, ctypes.c_double, pp]),
        "shm_host_rotate": (i32, [_P, _P, i32, pp]),
        "shm_host_conjugate": (i32, [_P, _P, pp]),
        "shm_host_multiply_i": (i32, [_P, _P, i32, pp]),
        "shm_host_to_shared": (i32, [_P, _P, _U32, pp]),
        "shm_host_slice": (i32, [_P, _P, _U32, _U32, pp]),
        "shm_host_ctpt_matmul": (i32, [_P, _P, ctypes.POINTER(ctypes.c_int64), _U32, ctypes.c_double, i32, pp]),
        "shm_host_ctpt_matmul_masked": (i32, [_P, _P, ctypes.POINTER(ctypes.c_int64), _U32, ctypes.c_double, dp, i32,
                                              pp]),
        "shm_host_from_shared": (i32, [_P, _P, pp]),
        "shm_boot_create": (i32, [_P, ctypes.c_double, _U32, pp]),
        "shm_boot_destroy": (None, [_P]),
        "shm_boot_galois_elts": (i32, [_P, ctypes.POINTER(_U32), _U32, ctypes.POINTER(_U32)]),
        "shm_boot_run": (i32, [_P, _P, _U32, pp]),
        "shm_boot_run_c2s_first": (i32, [_P, _P, pp]),
        "shm_boot_bert_layer": (i32, [_P, _P, ctypes.POINTER(_U32), dp, dp, ctypes.POINTER(ctypes.c_int), pp, dp]),
        "shm_boot_capture": (i32, [_P, _P, _U32, pp, pp]),
        "shm_boot_tune": (i32, [_P, _U32, _U32, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
        "shm_boot_get_split": (i32, [_P, ctypes.POINTER(ctypes.c_int)]),
        "shm_boot_set_split": (i32, [_P, ctypes.POINTER(ctypes.c_int)]),
        "shm_host_graph_launch": (i32, [_P]),
        "shm_host_graph_kernels": (ctypes.c_uint64, [_P]),
        "shm_host_graph_destroy": (None, [_P]),
        "shm_ct_write": (i32, [_P, _P, u64p]),
        "shm_host_encode": (i32, [_P, dp, dp, _U32, ctypes.c_double, ctypes.POINTER(ctypes.c_int64), i32]),
        "shm_slot_transform_selfcheck": (ctypes.c_double, [_U32]),
        "shm_ct_serialized_bytes": (i32, [_P, _P, ctypes.POINTER(ctypes.c_size_t)]),
        "shm_ct_serialize": (i32, [_P, _P, ctypes.c_void_p, ctypes.c_size_t]),
        "shm_ct_deserialize": (i32, [_P, ctypes.c_void_p, ctypes.c_size_t, pp]),
        "shm_host_save_keys": (i32, [_P, ctypes.c_char_p, i32]),
        "shm_host_load_keys": (i32, [_P, ctypes.c_char_p]),
        "shm_host_import_secret_text": (i32, [_P, ctypes.c_char_p]),
        "shm_host_export_secret_text": (i32, [_P, ctypes.c_char_p]),
        "shm_host_import_key": (i32, [_P, i32, _U32, u64p, ctypes.c_size_t]),
        "shm_host_chebyshev": (i32, [_P, _P, dp, _U32, ctypes.c_double, ctypes.c_double, pp]),
        "shm_host_gelu": (i32, [_P, _P, pp]),
        "shm_host_exp": (i32, [_P, _P, pp]),
        "shm_host_inverse": (i32, [_P, _P, _U32, pp]),
        "shm_host_inv_sqrt": (i32, [_P, _P, _U32, _U32, pp]),
        "shm_host_layernorm": (i32, [_P, _P, dp, dp, _U32, _U32, pp]),
        "shm_host_softmax": (i32, [_P, _P, ctypes.c_double, ctypes.c_double, _U32, pp]),
        "shm_host_softmax_attention": (i32, [_P, _P, ctypes.POINTER(ctypes.c_int), i32, _U32, pp]),
        "shm_host_ct_ct_matmul": (i32, [_P, _P, _P, _U32, _U32, pp]),
        "shm_host_ct_ct_matmul_diag": (i32, [_P, _P, _P, _U32, pp]),
        "shm_host_chebyshev_capture": (i32, [_P, _P, dp, _U32, ctypes.c_double, ctypes.c_double, pp, pp]),
        "shm_server_create": (i32, [_P, _P, ctypes.c_size_t, _U32, _U32, pp]),
        "shm_server_destroy": (None, [_P]),
        "shm_server_submit_rotate": (i32, [_P, _P, i32, ctypes.POINTER(ctypes.c_uint64)]),
        "shm_server_submit_matmul": (i32, [_P, _P, ctypes.POINTER(ctypes.c_int64), _U32, ctypes.c_double,
                                           ctypes.POINTER(ctypes.c_uint64)]),
        "shm_server_submit_bootstrap": (i32, [_P, _P, _U32, ctypes.POINTER(ctypes.c_uint64)]),
        "shm_server_wait": (i32, [_P, ctypes.c_uint64, pp, dp, ctypes.POINTER(_U32)]),
        "shm_server_set_paused": (i32, [_P, i32]),
        "shm_server_stats": (i32, [_P, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t),
                                   ctypes.POINTER(_U32), ctypes.POINTER(ctypes.c_uint64),
                                   ctypes.POINTER(ctypes.c_uint64)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _libs[path] = L
    return L


BERT_STAGES = ["Attention Block", "SelfOutput", "1st Bootstrapping", "LayerNorm1", "2nd Bootstrapping",
               "Intermediate Linear", "GELU", "Final Linear", "3rd Bootstrapping", "LayerNorm2", "4th Bootstrapping"]


class HostError(RuntimeError):
    pass


class Host:
    def __init__(self, log_n: int, primes=None, n_special: int = 0, hamming_weight: int = 192, seed: int = 0x5EED,
                 device: int = 0, lib: str | None = None, bits=None):
        self.lib = load(lib)
        h = _P()
        if primes is None:
            if bits is None:
                raise ValueError("give primes or bits")
            b = (ctypes.c_int * len(bits))(*bits)
            self._check(self.lib.shm_host_create_from_bits(ctypes.byref(h), log_n, b, len(bits), n_special, device,
                                                           hamming_weight, seed))
            pr = np.zeros(len(bits), dtype=np.uint64)
            self._check(self.lib.shm_host_primes(h, pr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        else:
            pr = np.ascontiguousarray(primes, dtype=np.uint64)
            self._check(self.lib.shm_host_create(ctypes.byref(h), log_n,
                                                 pr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(pr),
                                                 n_special, device, hamming_weight, seed))
        self._h = h
        self.primes = [int(p) for p in pr]
        self.log_n, self.n = log_n, 1 << log_n
        self.nq, self.np = len(pr) - n_special, n_special

    def _check(self, rc):
        if rc != 0:
            raise HostError(f"{rc}: {self.lib.shm_host_last_error().decode()}")

    def close(self):
        if getattr(self, "_h", None):
            self.lib.shm_host_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- keys
    def gen_relin_key(self):
        self._check(self.lib.shm_host_gen_relin_key(self._h))

    def gen_galois_keys(self, elts):
        e = (_U32 * len(elts))(*elts)
        self._check(self.lib.shm_host_gen_galois_keys(self._h, e, len(elts)))

    def gen_shared_keys(self, members: int, elts, hamming_weight: int = 192):
        e = (_U32 * len(elts))(*elts)
        self._check(self.lib.shm_host_gen_shared_keys(self._h, members, hamming_weight, e, len(elts)))

    def save_keys(self, path: str, with_secrets: bool = True):
        """Write the secrets (optional), relinearisation, Galois and shared-a keys as binary records."""
        self._check(self.lib.shm_host_save_keys(self._h, os.fsencode(path), 1 if with_secrets else 0))

    def load_keys(self, path: str):
        self._check(self.lib.shm_host_load_keys(self._h, os.fsencode(path)))

    def import_secret_text(self, path: str):
        """Take the secret from the reference's text format (NTT residues over Q*P, one per line)."""
        self._check(self.lib.shm_host_import_secret_text(self._h, os.fsencode(path)))

    def export_secret_text(self, path: str):
        self._check(self.lib.shm_host_export_secret_text(self._h, os.fsencode(path)))

    def import_key(self, words: np.ndarray, elt: int | None = None):
        """Install a key [dnum][2][QP][N]: the relinearisation key, or the Galois key of `elt`."""
        w = np.ascontiguousarray(words, dtype=np.uint64)
        self._check(self.lib.shm_host_import_key(self._h, 0 if elt is None else 1, elt or 0,
                                                 w.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), w.size))

    def deserialize(self, data: bytes) -> "Ct":
        """A ciphertext batch from one binary record (Ct.serialize)."""
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        return self._out(self.lib.shm_ct_deserialize, ctypes.cast(buf, ctypes.c_void_p), len(data))

    def galois_elt(self, step: int) -> int:
        return int(self.lib.shm_host_galois_elt(self._h, step))

    def synchronize(self):
        self._check(self.lib.shm_host_synchronize(self._h))

    def device_memory(self, reset_peak: bool = False) -> tuple[int, int]:
        """(bytes in use, peak bytes in use) of the host library's device pool."""
        used, peak = ctypes.c_size_t(), ctypes.c_size_t()
        self._check(self.lib.shm_host_device_memory(self._h, ctypes.byref(used), ctypes.byref(peak),
                                                    1 if reset_peak else 0))
        return used.value, peak.value

    # ---- ciphertexts
    def _out(self, fn, *args) -> "Ct":
        o = _P()
        self._check(fn(self._h, *args, ctypes.byref(o)))
        return Ct(self, o)

    def encrypt(self, z, scale: float, L: int) -> "Ct":
        z = np.atleast_2d(np.asarray(z, dtype=np.complex128))
        re = np.ascontiguousarray(z.real)
        im = np.ascontiguousarray(z.imag)
        dp = ctypes.POINTER(ctypes.c_double)
        return self._out(self.lib.shm_host_encrypt, re.ctypes.data_as(dp), im.ctypes.data_as(dp), z.shape[0],
                         z.shape[1], L, scale)

    def gen_public_key(self, seed: int = 0xE0C0):
        self._check(self.lib.shm_host_gen_public_key(self._h, seed))

    def encrypt_public(self, z, scale: float, L: int) -> "Ct":
        """Public-key encryption (encrypt_asymmetric); gen_public_key first."""
        z = np.atleast_2d(np.asarray(z, dtype=np.complex128))
        re = np.ascontiguousarray(z.real)
        im = np.ascontiguousarray(z.imag)
        dp = ctypes.POINTER(ctypes.c_double)
        return self._out(self.lib.shm_host_encrypt_public, re.ctypes.data_as(dp), im.ctypes.data_as(dp),
                         z.shape[0], z.shape[1], L, scale)

    def batch_input(self, X, scale: float, L: int) -> "Ct":
        """X [num_X][num_row][num_col] -> num_col ciphertexts in the column-interleaved packing (public key)."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        nx, nr, nc = X.shape
        dp = ctypes.POINTER(ctypes.c_double)
        return self._out(self.lib.shm_host_batch_input, X.ctypes.data_as(dp), nx, nr, nc, scale, L)

    def decrypt(self, ct: "Ct") -> np.ndarray:
        rows = ct.count * ct.members
        re = np.zeros((rows, self.n // 2))
        im = np.zeros((rows, self.n // 2))
        dp = ctypes.POINTER(ctypes.c_double)
        self._check(self.lib.shm_host_decrypt(self._h, ct._c, re.ctypes.data_as(dp), im.ctypes.data_as(dp)))
        return re + 1j * im

    def encode_coeffs(self, z, scale: float, on_host: bool = False) -> np.ndarray:
        """Integer coefficients of one slot vector: the device encoder, or the host FFT restatement."""
        z = np.asarray(z, dtype=np.complex128)
        re, im = np.ascontiguousarray(z.real), np.ascontiguousarray(z.imag)
        out = np.empty(self.n, dtype=np.int64)
        self._check(self.lib.shm_host_encode(self._h, re.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                             im.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(z), scale,
                                             out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), int(on_host)))
        return out

    def ct_from_host(self, data: np.ndarray, scale: float, shared: bool = False) -> "Ct":
        d = np.ascontiguousarray(data, dtype=np.uint64)
        count, size, L, _ = d.shape
        return self._out(self.lib.shm_ct_from_host, d.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), count, size,
                         L, scale, 1 if shared else 0)

    def ct_from_ptr(self, ptr: int, count: int, size: int, L: int, scale: float, shared: bool = False) -> "Ct":
        """Copy a batch from host memory at address `ptr` (e.g. a pinned buffer) to the device."""
        return self._out(self.lib.shm_ct_from_host, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint64)), count, size,
                         L, scale, 1 if shared else 0)

    def add(self, a, b):
        return self._out(self.lib.shm_host_add, a._c, b._c)

    def sub(self, a, b):
        return self._out(self.lib.shm_host_sub, a._c, b._c)

    def multiply(self, a, b):
        return self._out(self.lib.shm_host_multiply, a._c, b._c)

    def rescale(self, a):
        return self._out(self.lib.shm_host_rescale, a._c)

    def multiply_const(self, a, v: float):
        return self._out(self.lib.shm_host_multiply_const, a._c, v)

    def rotate(self, a, step: int):
        return self._out(self.lib.shm_host_rotate, a._c, step)

    def conjugate(self, a):
        return self._out(self.lib.shm_host_conjugate, a._c)

    def multiply_i(self, a, sign: int = 1):
        return self._out(self.lib.shm_host_multiply_i, a._c, sign)

    def slice(self, a, first: int = 0, count: int | None = None):
        """A device copy of ciphertexts [first, first + count) (the whole batch by default)."""
        return self._out(self.lib.shm_host_slice, a._c, first, a.count - first if count is None else count)

    def ctpt_matmul(self, X, W: np.ndarray, w_scale: float, tensor_cores: bool = True):
        W = np.ascontiguousarray(W, dtype=np.int64)
        return self._out(self.lib.shm_host_ctpt_matmul, X._c, W.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         W.shape[1], w_scale, 1 if tensor_cores else 0)

    def ctpt_matmul_masked(self, X, W: np.ndarray, w_scale: float, mask, tensor_cores: bool = True):
        """mask (N/2 slot values) times the ct-pt matmul X W: the masked projection, two levels."""
        W = np.ascontiguousarray(W, dtype=np.int64)
        m = np.ascontiguousarray(mask, dtype=np.float64)
        if m.shape != (self.n // 2,):
            raise ValueError("mask needs N/2 slot values")
        return self._out(self.lib.shm_host_ctpt_matmul_masked, X._c,
                         W.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), W.shape[1], w_scale,
                         m.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1 if tensor_cores else 0)

    def chebyshev(self, a, coeffs, lo: float, hi: float):
        """sum_k coeffs[k] T_k(u), u = (2 x - hi - lo) / (hi - lo), slot-wise, at the input's scale."""
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        return self._out(self.lib.shm_host_chebyshev, a._c, c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(c),
                         lo, hi)

    def gelu(self, a):
        """GELU by the reference's degree-24 Chebyshev series on [-19.5, 12.5] (6 levels)."""
        return self._out(self.lib.shm_host_gelu, a._c)

    def exp(self, a):
        """exp(x) as (1 + x/128)^128 (the softmax's exp, 8 levels)."""
        return self._out(self.lib.shm_host_exp, a._c)

    def inverse(self, a, iter: int):
        """1/x for x in (0, 2) as prod_{i <= iter} (1 + (1 - x)^(2^i)) (iter + 1 levels)."""
        return self._out(self.lib.shm_host_inverse, a._c, iter)

    def inv_sqrt(self, a, d_newt: int = 4, d_gold: int = 2):
        """1/sqrt(x) as LayerNorm's invert_sqrt: linear guess, Newton then Goldschmidt steps."""
        return self._out(self.lib.shm_host_inv_sqrt, a._c, d_newt, d_gold)

    def layernorm(self, a, gamma, beta, d_newt: int = 4, d_gold: int = 2):
        """LayerNorm over the batch's ciphertexts (one hidden column each): gamma_i (x_i - mean) / sqrt(var) + beta_i."""
        g = np.ascontiguousarray(gamma, dtype=np.float64)
        b = np.ascontiguousarray(beta, dtype=np.float64)
        if len(g) != a.count or len(b) != a.count:
            raise ValueError("gamma and beta need one value per ciphertext")
        dp = ctypes.POINTER(ctypes.c_double)
        return self._out(self.lib.shm_host_layernorm, a._c, g.ctypes.data_as(dp), b.ctypes.data_as(dp), d_newt, d_gold)

    def softmax(self, a, shift: float, sum_scale: float, iter: int):
        """e_i / sum_j e_j over the batch's ciphertexts, e_i = exp(x_i - shift) as (1 + (x_i - shift)/128)^128."""
        return self._out(self.lib.shm_host_softmax, a._c, shift, sum_scale, iter)

    def softmax_attention(self, a, bias_vec, input_num: int, iter: int):
        """The attention block's softmax with the reference's masks (bias_vec: one 0/1 per slot)."""
        b = np.ascontiguousarray(bias_vec, dtype=np.int32)
        if b.size != self.n // 2:
            raise ValueError("bias_vec needs one entry per slot")
        return self._out(self.lib.shm_host_softmax_attention, a._c, b.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                         input_num, iter)

    def ct_ct_matmul(self, X, W, rows: int, num_batch: int):
        """Column-packed ct-ct product: out_i = sum_j X_j * rot(W_j, i * num_batch), i < rows."""
        return self._out(self.lib.shm_host_ct_ct_matmul, X._c, W._c, rows, num_batch)

    def ct_ct_matmul_diag(self, X, W, num_batch: int):
        """Diagonal-packed ct-ct product (baby-step giant-step over X's diagonals), W.count outputs."""
        return self._out(self.lib.shm_host_ct_ct_matmul_diag, X._c, W._c, num_batch)

    def capture_chebyshev(self, ct, coeffs=None, lo: float = 0.0, hi: float = 0.0):
        """A CUDA graph of chebyshev(ct, coeffs, lo, hi) (GELU when coeffs is None) and the output
        batch every launch rewrites; write the next input into `ct` between launches."""
        o, g = _P(), _P()
        if coeffs is None:
            cp, n = None, 0
        else:
            c = np.ascontiguousarray(coeffs, dtype=np.float64)
            cp, n = c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(c)
        self._check(self.lib.shm_host_chebyshev_capture(self._h, ct._c, cp, n, lo, hi, ctypes.byref(o),
                                                        ctypes.byref(g)))
        return Graph(self, g, keep=ct), Ct(self, o)

    def to_shared(self, a, members: int):
        return self._out(self.lib.shm_host_to_shared, a._c, members)

    def from_shared(self, a):
        return self._out(self.lib.shm_host_from_shared, a._c)


class Ct:
    def __init__(self, host: Host, handle):
        self.host, self._c = host, handle
        c, s, L, sh = _U32(), _U32(), _U32(), ctypes.c_int()
        sc = ctypes.c_double()
        host._check(host.lib.shm_ct_info(handle, ctypes.byref(c), ctypes.byref(s), ctypes.byref(L), ctypes.byref(sc),
                                         ctypes.byref(sh)))
        self.count, self.size, self.level, self.scale, self.shared = c.value, s.value, L.value, sc.value, bool(sh.value)

    @property
    def members(self) -> int:
        return self.size - 1 if self.shared else 1

    def to_host(self) -> np.ndarray:
        out = np.empty((self.count, self.size, self.level, self.host.n), dtype=np.uint64)
        self.host._check(self.host.lib.shm_ct_to_host(self.host._h, self._c,
                                                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return out

    def to_ptr(self, ptr: int):
        """Copy the batch to host memory at address `ptr` (count * size * L * N words)."""
        self.host._check(self.host.lib.shm_ct_to_host(self.host._h, self._c,
                                                      ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint64))))

    def write_from_ptr(self, ptr: int):
        """Overwrite the batch's residues from host memory at `ptr` (the to_ptr layout)."""
        self.host._check(self.host.lib.shm_ct_write(self.host._h, self._c,
                                                    ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint64))))

    def serialize(self) -> bytes:
        """The batch as one binary record (header, residues, digest)."""
        n = ctypes.c_size_t()
        self.host._check(self.host.lib.shm_ct_serialized_bytes(self.host._h, self._c, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        self.host._check(self.host.lib.shm_ct_serialize(self.host._h, self._c, ctypes.cast(buf, ctypes.c_void_p),
                                                        n.value))
        return buf.raw

    def device_ptr(self) -> int:
        return int(self.host.lib.shm_ct_device_data(self._c) or 0)

    def close(self):
        if getattr(self, "_c", None):
            self.host.lib.shm_ct_destroy(self._c)
            self._c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Bootstrapper:
    def __init__(self, host: Host, scale: float = 2.0 ** 46, input_level: int = 4):
        self.host = host
        b = _P()
        host._check(host.lib.shm_boot_create(host._h, scale, input_level, ctypes.byref(b)))
        self._b = b
        self.scale, self.input_level = scale, input_level

    def galois_elts(self) -> list[int]:
        n = _U32()
        buf = (_U32 * 4096)()
        self.host._check(self.host.lib.shm_boot_galois_elts(self._b, buf, 4096, ctypes.byref(n)))
        return [int(buf[i]) for i in range(n.value)]

    def run(self, ct: Ct, members: int = 0) -> Ct:
        o = _P()
        self.host._check(self.host.lib.shm_boot_run(self._b, ct._c, members, ctypes.byref(o)))
        return Ct(self.host, o)

    def run_c2s_first(self, ct: Ct) -> Ct:
        """The original per-ciphertext C2S-first bootstrap (bootstrap_3)."""
        o = _P()
        self.host._check(self.host.lib.shm_boot_run_c2s_first(self._b, ct._c, ctypes.byref(o)))
        return Ct(self.host, o)

    def bert_layer(self, X: Ct, weights: dict, cfg: dict, bias_vec) -> tuple[Ct, dict]:
        """One BERT encoder layer (shm_boot_bert_layer) -> (output, {stage: seconds})."""
        d, F = cfg["hidden"], cfg["ffn"]
        order = [("Wq", d * d), ("bq", d), ("Wk", d * d), ("bk", d), ("Wv", d * d), ("bv", d), ("Wo", d * d),
                 ("bo", d), ("ln1_gamma", d), ("ln1_beta", d), ("Wi", d * F), ("bi", F), ("Wf", F * d), ("bf", d),
                 ("ln2_gamma", d), ("ln2_beta", d)]
        flat = np.concatenate([np.ascontiguousarray(weights[k], dtype=np.float64).reshape(-1) for k, n in order])
        assert flat.size == sum(n for _, n in order), "weight shapes"
        keys = ["hidden", "heads", "ffn", "num_X", "tokens", "input_num", "softmax_iter", "ln_newt", "ln_gold",
                "gelu_input_level", "ffn_chunk", "members", "boot_batch"]
        dims = (_U32 * len(keys))(*[int(cfg[k]) for k in keys])
        reals = np.array([cfg.get("w_scale", 2.0 ** 40), cfg.get("ln_var_scale", 64.0)], dtype=np.float64)
        bv = np.ascontiguousarray(bias_vec, dtype=np.int32)
        secs = np.zeros(22, dtype=np.float64)
        dp = ctypes.POINTER(ctypes.c_double)
        o = _P()
        self.host._check(self.host.lib.shm_boot_bert_layer(
            self._b, X._c, dims, reals.ctypes.data_as(dp), flat.ctypes.data_as(dp),
            bv.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(o), secs.ctypes.data_as(dp)))
        self.last_stage_peak_gb = dict(zip(BERT_STAGES, secs[11:].tolist()))
        return Ct(self.host, o), dict(zip(BERT_STAGES, secs[:11].tolist()))

    def tune(self, count: int, members: int = 0) -> list[dict]:
        """Autotune for batches of `count` (shm_boot_tune); generate Galois keys afterwards."""
        buf = ctypes.create_string_buffer(1 << 16)
        need = ctypes.c_size_t()
        self.host._check(self.host.lib.shm_boot_tune(self._b, count, members, buf, len(buf), ctypes.byref(need)))
        return json.loads(buf.value.decode())

    @property
    def split(self) -> list[int]:
        """BSGS baby-step counts of the six slot-transform layers (0 = default)."""
        g = (ctypes.c_int * 6)()
        self.host._check(self.host.lib.shm_boot_get_split(self._b, g))
        return list(g)

    @split.setter
    def split(self, g1):
        g = (ctypes.c_int * 6)(*g1)
        self.host._check(self.host.lib.shm_boot_set_split(self._b, g))

    def capture(self, ct: Ct, members: int = 0) -> tuple["Graph", Ct]:
        """A CUDA graph of run(ct, members) and the output batch every launch rewrites;
        write the next input into `ct` (Ct.write_from_ptr) between launches."""
        o, g = _P(), _P()
        self.host._check(self.host.lib.shm_boot_capture(self._b, ct._c, members, ctypes.byref(o), ctypes.byref(g)))
        return Graph(self.host, g, keep=ct), Ct(self.host, o)

    def close(self):
        if getattr(self, "_b", None):
            self.host.lib.shm_boot_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """A recorded batch of device work (shm_host_graph); launch() replays it on the host's stream."""

    def __init__(self, host: Host, handle, keep=None):
        self.host, self._g, self._keep = host, handle, keep  # the captured input must outlive the graph

    @property
    def kernels(self) -> int:
        return int(self.host.lib.shm_host_graph_kernels(self._g))

    def launch(self):
        self.host._check(self.host.lib.shm_host_graph_launch(self._g))

    def close(self):
        if getattr(self, "_g", None):
            self.host.lib.shm_host_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The serving loop (shm_server_*): HBM-budget admission onto `slots` concurrent
    streams, continuous batching of queued jobs of the same kind and shape.  Submitting
    a ciphertext hands it over (the Ct object is emptied)."""

    def __init__(self, host: Host, boot: Bootstrapper | None = None, hbm_budget: int = 64 << 30, slots: int = 2,
                 max_merge: int = 64):
        self.host = host
        s = _P()
        host._check(host.lib.shm_server_create(host._h, boot._b if boot else None, hbm_budget, slots, max_merge,
                                               ctypes.byref(s)))
        self._s = s

    def _submit(self, fn, ct: Ct, *args) -> int:
        job = ctypes.c_uint64()
        handle, ct._c = ct._c, None  # ownership moves to the server (freed even on error)
        self.host._check(fn(self._s, handle, *args, ctypes.byref(job)))
        return int(job.value)

    def submit_rotate(self, ct: Ct, step: int) -> int:
        return self._submit(self.host.lib.shm_server_submit_rotate, ct, step)

    def submit_matmul(self, ct: Ct, W: np.ndarray, w_scale: float) -> int:
        W = np.ascontiguousarray(W, dtype=np.int64)
        if W.shape[0] != ct.count:
            raise ValueError("W must be [n_in][n_out]")
        return self._submit(self.host.lib.shm_server_submit_matmul, ct,
                            W.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), W.shape[1], w_scale)

    def submit_bootstrap(self, ct: Ct, members: int = 0) -> int:
        return self._submit(self.host.lib.shm_server_submit_bootstrap, ct, members)

    def wait(self, job: int):
        """(result Ct, (t_submit, t_start, t_end), jobs that shared its launches)"""
        o = _P()
        t = (ctypes.c_double * 3)()
        b = _U32()
        self.host._check(self.host.lib.shm_server_wait(self._s, job, ctypes.byref(o), t, ctypes.byref(b)))
        return Ct(self.host, o), (t[0], t[1], t[2]), int(b.value)

    def pause(self, paused: bool = True):
        self.host._check(self.host.lib.shm_server_set_paused(self._s, 1 if paused else 0))

    def resume(self):
        self.pause(False)

    def stats(self) -> dict:
        v = [ctypes.c_size_t(), ctypes.c_size_t(), _U32(), ctypes.c_uint64(), ctypes.c_uint64()]
        self.host._check(self.host.lib.shm_server_stats(self._s, *[ctypes.byref(x) for x in v]))
        return dict(zip(("budget", "peak_admitted", "max_inflight", "batches", "jobs"), (x.value for x in v)))

    def close(self):
        if getattr(self, "_s", None):
            self.host.lib.shm_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def slot_transform_selfcheck(log_slots: int, lib: str | None = None) -> float:
    return float(load(lib).shm_slot_transform_selfcheck(log_slots))


def bias_vec(lengths, num_X: int, num_row: int, lib: str | None = None) -> np.ndarray:
    """The valid-slot mask of the column-interleaved packing (Batch_encode_encrypt.cuh:45-56)."""
    ln = np.ascontiguousarray(lengths, dtype=np.int32)
    out = np.zeros(num_X * num_row, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    L = load(lib)
    if L.shm_host_bias_vec(ln.ctypes.data_as(ip), num_X, num_row, out.ctypes.data_as(ip)) != 0:
        raise HostError(L.shm_host_last_error().decode())
    return out
