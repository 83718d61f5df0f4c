"""Scale-exact CKKS evaluator over batches of ciphertexts.

A ``Ct`` is a batch of ciphertexts [n][2][L][N] that share one level L and one
scale.  The scale is tracked exactly (float64 products and quotients of the
primes and encoded constants), never assumed to stay at a nominal 2^k: adding
ciphertexts whose scales differ is an error, and ``adjust`` brings a
ciphertext to a target (level, scale) pair by one constant multiply.

Counterpart of the reference's moai::Evaluator / CKKSEvaluator level and scale
handling (src/include/source/ckks_evaluator_parallel.cuh:245-360,
ckks_evaluator_parallel.cu:548-590: multiply_const, add_const, the
*_reduced_error level alignment).  All ring work goes through the backend
(backend.GpuBackend: the CUDA library).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .encoder import Encoder


@dataclass
class Ct:
    data: object  # backend array [n][2][L][N]
    scale: float

    @property
    def level(self) -> int:
        return int(self.data.shape[-2])

    @property
    def batch(self) -> int:
        return int(self.data.shape[0])

    def like(self, data, scale: float | None = None):
        """A ciphertext of the same kind holding `data`."""
        return type(self)(data, self.scale if scale is None else scale)


@dataclass
class ShCt(Ct):
    """Shared-a groups [G][n + 1][L][N] = (b_0 .. b_{n-1}, a) with b_i + a s'_i ~ m_i
    (SharedACiphertextBatch, src/include/source/bootstrapping/SharedACiphertext.cuh:22-99).
    Linear operations, plaintext products, rescale and modraise act on all n + 1
    polynomials alike; rotations are Sh-Rots with the Sh-Galois keys."""

    @property
    def members(self) -> int:
        return int(self.data.shape[1]) - 1


@dataclass
class SharedKeys:
    """Keys of one shared-a group size: Sh-Galois keys by element ([dnum][n + 1][QP][N]),
    the format key ([n][n + 1][QP][N]) and the n backward switching keys s'_i -> s."""
    galois: dict = field(default_factory=dict)
    fmt: object = None
    backward: list = field(default_factory=list)


class ScaleMismatch(ValueError):
    pass


class Evaluator:
    def __init__(self, backend, relin_key=None, galois_keys=None):
        self.be = backend
        self.relin_key = relin_key
        self.galois_keys = galois_keys if galois_keys is not None else {}
        self.primes = backend.primes
        self.nq = backend.nq
        self.enc = Encoder(backend.log_n)
        self._mono = None
        self.shared = SharedKeys()

    # ---------------- helpers ----------------
    def _residues(self, k: int, L: int) -> np.ndarray:
        return np.array([k % self.primes[i] for i in range(L)], dtype=np.uint64)

    def drop(self, a: Ct, L: int) -> Ct:
        if L > a.level:
            raise ValueError("cannot raise the level by dropping")
        return a.like(self.be.drop(a.data, L))

    @staticmethod
    def same_scale(s1: float, s2: float, rel: float = 1e-11) -> bool:
        return abs(s1 - s2) <= rel * max(abs(s1), abs(s2))

    def _align(self, a: Ct, b: Ct):
        L = min(a.level, b.level)
        a2, b2 = self.drop(a, L), self.drop(b, L)
        if not self.same_scale(a.scale, b.scale):
            raise ScaleMismatch(f"scale mismatch {a.scale!r} vs {b.scale!r}")
        return a2, b2

    # ---------------- linear ops ----------------
    def add(self, a: Ct, b: Ct) -> Ct:
        a, b = self._align(a, b)
        return a.like(self.be.add(a.data, b.data))

    def sub(self, a: Ct, b: Ct) -> Ct:
        a, b = self._align(a, b)
        return a.like(self.be.sub(a.data, b.data))

    def neg(self, a: Ct) -> Ct:
        return a.like(self.be.neg(a.data))

    def mul_int(self, a: Ct, k: int) -> Ct:
        """Multiply by an integer exactly (scale unchanged, no level)."""
        return a.like(self.be.mul_scalar(a.data, self._residues(int(k), a.level)))

    def add_const(self, a: Ct, c: float) -> Ct:
        """Add c to every slot (no level)."""
        if isinstance(a, ShCt):
            raise TypeError("add_const on shared-a groups is not supported")
        k = int(round(c * a.scale))
        return Ct(self.be.add_scalar(a.data, self._residues(k, a.level)), a.scale)

    def rescale(self, a: Ct) -> Ct:
        q = self.primes[a.level - 1]
        return a.like(self.be.rescale(a.data), a.scale / q)

    def mul_const(self, a: Ct, c: float, target_scale: float | None = None) -> Ct:
        """Multiply by a real constant; one level.  The constant is encoded so the
        result has exactly `target_scale` (default: the input's scale)."""
        target = a.scale if target_scale is None else target_scale
        q = self.primes[a.level - 1]
        T = target * q / a.scale
        k = int(round(c * T))
        out = self.be.mul_scalar(a.data, self._residues(k, a.level))
        return a.like(self.be.rescale(out), target)

    def mul_const_unscaled(self, a: Ct, c: float, T: float):
        """a * round(c * T) without rescale; the result's scale is a.scale * T (for fused sums)."""
        k = int(round(c * T))
        return a.like(self.be.mul_scalar(a.data, self._residues(k, a.level)), a.scale * T)

    def adjust(self, a: Ct, level: int, scale: float) -> Ct:
        """Bring `a` to (level, scale): a pure drop when the scale already matches,
        otherwise a drop to level+1 and one exact constant multiply."""
        if a.level == level and self.same_scale(a.scale, scale):
            return a.like(a.data, scale)
        if a.level <= level:
            if self.same_scale(a.scale, scale):
                return self.drop(a, level) if a.level > level else a
            raise ValueError("cannot adjust the scale without a spare level")
        return self.mul_const(self.drop(a, level + 1), 1.0, scale)

    # ---------------- multiplicative ops ----------------
    def mul(self, a: Ct, b: Ct, rescale: bool = True) -> Ct:
        L = min(a.level, b.level)
        a2, b2 = self.drop(a, L), self.drop(b, L)
        t = self.be.tensor(a2.data, b2.data)
        r = Ct(self.be.relin(t, self.relin_key), a.scale * b.scale)
        return self.rescale(r) if rescale else r

    def square(self, a: Ct) -> Ct:
        return self.mul(a, a)

    # ---------------- slot permutations ----------------
    def galois_elt(self, step: int) -> int:
        n2 = 2 * self.be.n
        slots = self.be.n // 2
        if step == 0:
            return n2 - 1
        s = step % slots
        return pow(5, s, n2)

    def _keys_for(self, a: Ct, elts):
        table = self.shared.galois if isinstance(a, ShCt) else self.galois_keys
        for e in elts:
            if e not in table:
                kind = "Sh-Galois" if isinstance(a, ShCt) else "Galois"
                raise ValueError(f"{kind} key for element {e} not present")
        return [table[e] for e in elts]

    def _automorphisms(self, a: Ct, elts) -> list:
        keys = self._keys_for(a, elts)
        if isinstance(a, ShCt):
            res = self.be.sh_rotate_many(a.data, elts, keys)
        elif len(elts) == 1:
            res = [self.be.apply_galois(a.data, elts[0], keys[0])]
        else:
            res = self.be.apply_galois_many(a.data, elts, keys)
        return [a.like(r) for r in res]

    def rotate(self, a: Ct, step: int) -> Ct:
        if step % (self.be.n // 2) == 0:
            return a
        return self._automorphisms(a, [self.galois_elt(step)])[0]

    def rotate_many(self, a: Ct, steps) -> dict:
        """Rotations of the same ciphertext by several steps with one hoisted ModUp."""
        steps = [s for s in steps if s % (self.be.n // 2)]
        if not steps:
            return {}
        return dict(zip(steps, self._automorphisms(a, [self.galois_elt(s) for s in steps])))

    def conjugate(self, a: Ct) -> Ct:
        return self._automorphisms(a, [2 * self.be.n - 1])[0]

    # ---------------- shared-a format switches ----------------
    def to_shared(self, a: Ct, n: int) -> ShCt:
        """FmtSwitch forward: groups of n consecutive ciphertexts -> shared-a groups."""
        if a.batch % n:
            raise ValueError("batch is not a multiple of the group size")
        return ShCt(self.be.fmt_forward(a.data, n, self.shared.fmt), a.scale)

    def from_shared(self, a: ShCt) -> Ct:
        """FmtSwitch backward: shared-a groups -> ordinary ciphertexts under s."""
        return Ct(self.be.fmt_backward(a.data, self.shared.backward), a.scale)

    def monomial_half(self):
        """NTT form of X^(N/2) over all chain primes: multiplying by it multiplies
        every slot by i (omega_j^(N/2) = i for all slots), exactly and at no level."""
        if self._mono is None:
            c = np.zeros(self.be.n, dtype=np.int64)
            c[self.be.n // 2] = 1
            t = self.be.from_host(self.enc.to_rns(c, self.primes[: self.nq]))
            self._mono = self.be.ntt_fwd(t)
        return self._mono

    def mul_i(self, a: Ct, sign: int = 1) -> Ct:
        out = a.like(self.be.mul_plain(a.data, self.monomial_half()[: a.level]))
        return out if sign > 0 else self.neg(out)

    # ---------------- plaintexts ----------------
    def encode_ntt(self, z, scale: float, L: int):
        """Plaintext [L][N] in NTT form with slots z * scale."""
        t = self.be.from_host(self.enc.to_rns(self.enc.encode(z, scale), self.primes[:L]))
        return self.be.ntt_fwd(t)
