"""CKKS canonical-embedding encoder (FP64, host).

Slot j of a plaintext m(X) (degree < N, n = N/2 slots) is m(omega_j) / scale with
omega_j = exp(2*pi*i * 5^j / 2N): the slot order of the reference encoder
(thirdparty/phantom-fhe/src/ckks.cu:20-87, rotation group 5^j), under which the
automorphism X -> X^(5^s) rotates the slots left by s.

encode:  m_k = round((2 * scale / N) * Re(sum_j z_j * omega_j^-k)), one length-2N FFT.
decode:  z_j = (sum_k m_k * omega_j^k) / scale, one length-2N inverse FFT.

A constant vector w * ones encodes to the single coefficient round(w * scale)
(the reference's moai::Encoder::encode(double), ckks_evaluator_parallel.cuh:73-92;
the golden fixtures confirm the reference rounds exactly this way).
"""
from __future__ import annotations

import numpy as np


class Encoder:
    def __init__(self, log_n: int):
        self.log_n = log_n
        self.N = 1 << log_n
        self.n = self.N // 2
        self.M = 2 * self.N
        self.exps = np.array([pow(5, j, self.M) for j in range(self.n)], dtype=np.int64)

    def encode_float(self, z, scale: float) -> np.ndarray:
        """Unrounded real coefficients (float64) of the polynomial with slots z * scale."""
        z = np.asarray(z, dtype=np.complex128)
        if z.size != self.n:
            full = np.zeros(self.n, dtype=np.complex128)
            full[: z.size] = z
            z = full
        A = np.zeros(self.M, dtype=np.complex128)
        A[self.exps] = z
        f = np.fft.fft(A)[: self.N]
        return (2.0 * scale / self.N) * f.real

    def encode(self, z, scale: float) -> np.ndarray:
        """Integer coefficients (int64; |coefficient| < 2^62 required)."""
        c = np.rint(self.encode_float(z, scale))
        if np.abs(c).max(initial=0) >= 2.0 ** 62:
            raise ValueError("encoded values are too large")
        return c.astype(np.int64)

    def decode(self, coeffs, scale: float) -> np.ndarray:
        m = np.zeros(self.M, dtype=np.float64)
        m[: self.N] = np.asarray(coeffs, dtype=np.float64)
        B = np.fft.ifft(m) * self.M
        return B[self.exps] / scale

    @staticmethod
    def to_rns(coeffs: np.ndarray, primes) -> np.ndarray:
        """Signed integer coefficients -> [L][N] residues."""
        c = np.asarray(coeffs, dtype=np.int64)
        return np.stack([np.remainder(c, np.int64(q)).astype(np.uint64) for q in primes])

    @staticmethod
    def centered(limb0: np.ndarray, q0: int) -> np.ndarray:
        """Residues mod q0 -> centred signed values (float64)."""
        v = limb0.astype(np.float64)
        return np.where(limb0 > np.uint64(q0 // 2), v - float(q0), v)
