"""Loader for the reference golden fixtures and the rebuild of their inputs.

Every record of ``golden_<set>.json`` is an output of the reference evaluator
run on inputs drawn from the counter generator ``oracle.oracle.fill`` with a
fixed tag (see oracle/ref_golden.cu).  ``GoldenSet`` rebuilds those inputs and
keys and checks an array against a record (checksum + first 8 coefficients of
every limb).
"""
from __future__ import annotations

import json
import os

import numpy as np

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


class GoldenSet:
    def __init__(self, name: str):
        with open(os.path.join(HERE, f"golden_{name}.json")) as f:
            self.doc = json.load(f)
        p = self.doc["params"]
        self.name = name
        self.log_n = p["log_n"]
        self.n = 1 << self.log_n
        self.nq, self.np, self.dnum = p["nq"], p["np"], p["dnum"]
        self.primes = np.array([int(x) for x in p["primes"]], dtype=np.uint64)
        self.L = self.nq

    # ---- inputs --------------------------------------------------------
    def ct(self, tag: int, limbs: int | None = None) -> np.ndarray:
        L = self.L if limbs is None else limbs
        rows = list(self.primes[:L]) * 2
        return O.fill(tag, (2, L, self.n), rows)

    def plain(self, tag: int) -> np.ndarray:
        return O.fill(tag, (self.L, self.n), list(self.primes[: self.L]))

    def key(self, tag: int) -> np.ndarray:
        """[dnum][2][QP][N]; digit d drawn with tag + d."""
        rows = list(self.primes) * 2
        qp = len(self.primes)
        return np.stack([O.fill(tag + d, (2, qp, self.n), rows) for d in range(self.dnum)])

    def relin_key(self):
        return self.key(100)

    def galois_key(self, elt: int):
        return self.key(300 if elt == 5 else 200)

    # ---- records -------------------------------------------------------
    def record(self, name: str):
        return self.doc[name]

    def matches(self, name: str, arr: np.ndarray) -> tuple[bool, str]:
        rec = self.doc[name]
        a = np.ascontiguousarray(arr, dtype=np.uint64).reshape(-1, self.n)
        if a.shape[0] != rec["rows"]:
            return False, f"{name}: rows {a.shape[0]} != {rec['rows']}"
        head = np.array([[int(x) for x in r] for r in rec["head"]], dtype=np.uint64)
        if not np.array_equal(a[:, :8], head):
            bad = np.argwhere(a[:, :8] != head)[0]
            return False, f"{name}: head mismatch at row {bad[0]} col {bad[1]}: {a[bad[0], bad[1]]} != {head[bad[0], bad[1]]}"
        cs = O.checksum(a)
        if cs != rec["checksum"]:
            return False, f"{name}: checksum {cs} != {rec['checksum']}"
        return True, "ok"

    def ctpt_weights(self):
        """Integer weights the reference encoder produced, [n_in][n_out]."""
        cols = []
        o = 0
        while f"ctpt_wint_{o}" in self.doc:
            cols.append([int(x) for x in self.doc[f"ctpt_wint_{o}"]])
            o += 1
        return np.array(cols, dtype=np.int64).T

    def ctpt_inputs(self):
        n_in = self.ctpt_weights().shape[0]
        return np.stack([self.ct(20 + j) for j in range(n_in)])


class SharedGoldenSet(GoldenSet):
    """Records of ``golden_shared_<set>.json`` (oracle/ref_golden.cu, mode ``shared``): the
    reference's FmtSwitch forward / backward, Sh-Rot, shared batch rescale / modraise /
    multiply_plain / add, and a complex slot-vector encode, with their inputs rebuilt here in this
    library's layouts."""

    def __init__(self, name: str):
        super().__init__("shared_" + name)
        self.qp = self.nq + self.np

    def batch(self, tag: int, n: int, L: int) -> np.ndarray:
        """A shared-a group [n + 1][L][N] = (b_0 .. b_{n-1}, a): b_i drawn with tag + i, a with tag + 9."""
        rows = list(self.primes[:L])
        return np.stack([O.fill(tag + i, (L, self.n), rows) for i in range(n)] + [O.fill(tag + 9, (L, self.n), rows)])

    def cts(self, tag: int, n: int, L: int) -> np.ndarray:
        """n ciphertexts [n][2][L][N], ciphertext j drawn with tag + j."""
        return np.stack([self.ct(tag + j, L) for j in range(n)])

    def fmt_key(self, n: int, L: int) -> np.ndarray:
        """The format key [n][n + 1][QP][N] = (B_fmt[j][0..n-1], a_fmt[j]); the reference holds it in the
        QlP basis (FmtSwitch.cuh:31-40), whose rows go to this layout's Ql and P rows."""
        qlp = list(self.primes[:L]) + list(self.primes[self.nq:])
        key = np.zeros((n, n + 1, self.qp, self.n), dtype=np.uint64)
        for j in range(n):
            for i in range(n + 1):
                tag = 500 + j * n + i if i < n else 400 + j
                v = O.fill(tag, (L + self.np, self.n), qlp)
                key[j, i, :L] = v[:L]
                key[j, i, self.nq:] = v[L:]
        return key

    def backward_keys(self, n: int) -> list[np.ndarray]:
        """n key-switching keys [dnum][2][QP][N]; key i digit d drawn with tag 600 + 10 i + d."""
        return [self.key(600 + 10 * i) for i in range(n)]

    def shrot_key(self, n: int) -> np.ndarray:
        """Sh-Galois key [dnum][n + 1][QP][N] = (B_{d,0..n-1}, A_d); the reference's A_d has tag 700 + d and
        B_{d,i} tag 800 + d n + i (ShRotate.cuh:25-36)."""
        rows = list(self.primes)
        return np.stack([np.stack([O.fill(800 + d * n + i, (self.qp, self.n), rows) for i in range(n)]
                                  + [O.fill(700 + d, (self.qp, self.n), rows)]) for d in range(self.dnum)])

    def plain_at(self, tag: int, L: int) -> np.ndarray:
        return O.fill(tag, (L, self.n), list(self.primes[:L]))

    def slots(self) -> np.ndarray:
        """The encoded slot vector: unit(12, j) + i unit(13, j), unit = a 53-bit integer times 2^-52 minus 1."""
        j = np.arange(self.n // 2, dtype=np.uint64)
        re = (O.sm64((np.uint64(12) << np.uint64(40)) + j) >> np.uint64(11)).astype(np.float64) * 2.0 ** -52 - 1.0
        im = (O.sm64((np.uint64(13) << np.uint64(40)) + j) >> np.uint64(11)).astype(np.float64) * 2.0 ** -52 - 1.0
        return re + 1j * im

    def encode_coeffs(self) -> tuple[float, int, np.ndarray]:
        rec = self.doc["encode_z_coeffs"]
        return 2.0 ** rec["scale_log2"], rec["stride"], np.array([int(x) for x in rec["values"]], dtype=np.int64)


def exact_coefficient(z: np.ndarray, k: int, scale: float, log_n: int) -> float:
    """Coefficient k of the canonical-embedding encode of slot vector z (slot j at the root
    exp(i pi 5^j / N)) before rounding, in extended precision: (2/N) sum_j Re(z_j w^(-k 5^j)) * scale."""
    n = 1 << log_n
    m = 2 * n
    e = np.ones(n // 2, dtype=np.int64)
    for j in range(1, n // 2):
        e[j] = (e[j - 1] * 5) % m
    ang = np.arccos(np.longdouble(-1)) * ((e * k) % m).astype(np.longdouble) / np.longdouble(n)
    zr = z.real.astype(np.longdouble)
    zi = z.imag.astype(np.longdouble)
    # Re(z w^-a) = zr cos(a) + zi sin(a)
    s = np.sum(zr * np.cos(ang) + zi * np.sin(ang))
    return float(s * np.longdouble(2.0) / np.longdouble(n) * np.longdouble(scale))


def c_round(x: np.ndarray) -> np.ndarray:
    """C's round(): halves away from zero."""
    return np.sign(x) * np.floor(np.abs(x) + 0.5)
