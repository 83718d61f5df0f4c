"""Loader of the in-tree CUDA library ``shmoai_b200/_build/libshmoai_b200.so``.

There is no fallback: if the library is missing or does not load, importing
the package's GPU entry points raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libshmoai_b200.so")
CSRC = os.path.join(HERE, "csrc")

SHM_OK = 0
_lib = None

_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_SZ = ctypes.c_size_t


def build(jobs: int = 8) -> str:
    """Compile the CUDA library for sm_100a and the C++ host library over it, in place
    (nvcc / g++; no GPU needed)."""
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", CSRC], check=True)
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "host")], check=True)
    return LIB_PATH


def _declare(L):
    sig = {
        "shm_context_create": (ctypes.c_int, [ctypes.POINTER(_P), _U32, ctypes.POINTER(ctypes.c_int), _U32, _U32,
                                              ctypes.c_int]),
        "shm_context_create_from_primes": (ctypes.c_int, [ctypes.POINTER(_P), _U32,
                                                          ctypes.POINTER(ctypes.c_uint64), _U32, _U32, ctypes.c_int]),
        "shm_context_destroy": (None, [_P]),
        "shm_context_info": (ctypes.c_int, [_P] + [ctypes.POINTER(_U32)] * 4),
        "shm_context_primes": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64)]),
        "shm_last_error": (ctypes.c_char_p, []),
        "shm_kernel_launches": (ctypes.c_uint64, []),
        "shm_ntt_forward": (ctypes.c_int, [_P, _P, _U32, _U32, _P]),
        "shm_ntt_inverse": (ctypes.c_int, [_P, _P, _U32, _U32, _P]),
        "shm_add": (ctypes.c_int, [_P, _P, _P, _P, _U32, _U32, _P]),
        "shm_sub": (ctypes.c_int, [_P, _P, _P, _P, _U32, _U32, _P]),
        "shm_negate": (ctypes.c_int, [_P, _P, _P, _U32, _U32, _P]),
        "shm_multiply_plain": (ctypes.c_int, [_P, _P, _P, _P, _U32, _U32, _P]),
        "shm_multiply": (ctypes.c_int, [_P, _P, _P, _P, _U32, _U32, _P]),
        "shm_rescale_workspace_bytes": (_SZ, [_P, _U32, _U32]),
        "shm_rescale": (ctypes.c_int, [_P, _P, _P, _U32, _U32, _P, _SZ, _P]),
        "shm_keyswitch_workspace_bytes": (_SZ, [_P, _U32, _U32]),
        "shm_keyswitch": (ctypes.c_int, [_P, _P, _P, _P, _U32, _U32, _P, _SZ, _P]),
        "shm_relinearize": (ctypes.c_int, [_P, _P, _P, _P, _U32, _U32, _P, _SZ, _P]),
        "shm_apply_galois": (ctypes.c_int, [_P, _P, _U32, _P, _P, _U32, _U32, _P, _SZ, _P]),
        "shm_galois_elt_from_step": (_U32, [_P, ctypes.c_int]),
        "shm_apply_galois_hoisted_workspace_bytes": (_SZ, [_P, _U32, _U32]),
        "shm_apply_galois_hoisted": (ctypes.c_int, [_P, _P, _U32, ctypes.POINTER(_U32), ctypes.POINTER(_P),
                                                    ctypes.POINTER(_P), _U32, _U32, _P, _SZ, _P]),
        "shm_rotate": (ctypes.c_int, [_P, _P, ctypes.c_int, _P, _P, _U32, _U32, _P, _SZ, _P]),
        "shm_multiply_scalar": (ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_uint64), _P, _U32, _U32, _P]),
        "shm_add_scalar": (ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_uint64), _P, _U32, _U32, _P]),
        "shm_multiply_plain_accumulate": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), _U32, _P, _U32,
                                                         _U32, ctypes.c_int, _P]),
        "shm_linear_combination": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(_U32),
                                                  ctypes.POINTER(ctypes.c_uint64), _U32, ctypes.POINTER(ctypes.c_uint64),
                                                  _P, _U32, _U32, _P]),
        "shm_modraise_workspace_bytes": (_SZ, [_P, _U32]),
        "shm_modraise": (ctypes.c_int, [_P, _P, _P, _U32, _U32, _P, _SZ, _P]),
        "shm_drop_limbs": (ctypes.c_int, [_P, _P, _P, _U32, _U32, _U32, _P]),
        "shm_ctpt_matmul_workspace_bytes": (_SZ, [_P, _U32, _U32, _U32]),
        "shm_ctpt_matmul_cuda_core": (ctypes.c_int, [_P, _P, _P, _P, _U32, _U32, _U32, _P]),
        "shm_ctpt_matmul": (ctypes.c_int, [_P, _P, _P, _P, _U32, _U32, _U32, _P, _SZ, _P]),
        "shm_shared_rotate_workspace_bytes": (_SZ, [_P, _U32, _U32, _U32]),
        "shm_shared_rotate_one_workspace_bytes": (_SZ, [_P, _U32, _U32, _U32]),
        "shm_shared_rotate": (ctypes.c_int, [_P, _P, _U32, _U32, _U32, _P, _P, _U32, _P, _SZ, _P]),
        "shm_shared_rotate_hoisted": (ctypes.c_int, [_P, _P, _U32, _U32, _U32, ctypes.POINTER(_U32),
                                                     ctypes.POINTER(_P), ctypes.POINTER(_P), _U32, _P, _SZ, _P]),
        "shm_fmt_switch_forward_workspace_bytes": (_SZ, [_P, _U32, _U32, _U32]),
        "shm_fmt_switch_forward": (ctypes.c_int, [_P, _P, _U32, _U32, _P, _P, _U32, _P, _SZ, _P]),
        "shm_fmt_switch_backward_workspace_bytes": (_SZ, [_P, _U32, _U32, _U32]),
        "shm_fmt_switch_backward": (ctypes.c_int, [_P, _P, _U32, _U32, ctypes.POINTER(_P), _P, _U32, _P, _SZ,
                                                   _P]),
        "shm_stream_create": (ctypes.c_int, [_P, ctypes.POINTER(_P)]),
        "shm_stream_destroy": (ctypes.c_int, [_P, _P]),
        "shm_graph_begin": (ctypes.c_int, [_P, _P]),
        "shm_graph_end": (ctypes.c_int, [_P, _P, ctypes.POINTER(_P)]),
        "shm_graph_launch": (ctypes.c_int, [_P, _P]),
        "shm_graph_kernels": (ctypes.c_uint64, [_P]),
        "shm_graph_destroy": (None, [_P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def lib():
    """The loaded library; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"shmoai_b200 CUDA library not built: {LIB_PATH} (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return [n for n in dir(lib()) if n.startswith("shm_")]


class ShmError(RuntimeError):
    pass


def check(rc: int):
    if rc != SHM_OK:
        msg = lib().shm_last_error()
        raise ShmError(f"shmoai_b200 error {rc}: {msg.decode() if msg else ''}")
