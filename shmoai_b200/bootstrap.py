"""S2C-first CKKS bootstrapping over batches of ciphertexts.

Pipeline (the reference's BatchBootstrapper::bootstrap_ordinary_s2c_first,
src/include/source/bootstrapping/BatchBootstrap.cuh:674-704, input at 4 primes):

  SlotToCoeff (3 BSGS layers, 4 -> 1 primes; amplitude factor F on the last layer)
  -> ModRaise (1 -> n_q primes, scale := q0)
  -> CoeffToSlot (3 BSGS layers, n_q -> n_q - 3; the 1/(2K) EvalMod input factor folded in)
  -> real / imaginary split with ONE conjugation (w + conj w, -i (w - conj w))
  -> EvalMod on both halves as one batch: Chebyshev interpolant of
     cos(2 pi (K x - 1/4) / 2^r) (degree 47, K = 25) by baby-step giant-step,
     r = 3 double-angle steps, giving sin(2 pi t); the final constant
     q0 / (2 pi Delta F) and the scale Delta are reached through exact scale
     targets, not an extra level
  -> recombination re + i * im (i = the monomial X^(N/2), free).

Linear transforms: the slot-to-coefficient map V (V_jk = omega_j^k, slot order
5^j) factors, after a bit reversal that both directions absorb, into log2(n)
radix-2 butterfly stages; stages are grouped 5/5/5 (for n = 2^15) into three
sparse matrices with at most 63 diagonals each, applied by baby-step
giant-step with pre-rotated diagonals, one multiply-plain-accumulate per giant
step and one rescale per layer.  Diagonal plaintexts are encoded once and stay
resident on the device (the reference re-encodes them on every call,
SharedACoeffToSlot.cu:50-57).

Reference parameters (test_shared_a.cuh:1208-1250): N = 2^16, Q = [51] + 20x[46]
+ 14x[51], P = 5x[51], Delta = 2^46, h = 192, F = 1/16 (Bootstrapper.cuh:31).
EvalMod here uses degree 47 with three double angles where the reference uses a
degree-59 Remez fit with two (NTL-generated, ModularReducer.cu:40-54): the
Chebyshev interpolant with two double angles leaves ~2e-7 error, too much for
the 2e-5 target after the x512 amplitude correction, three give ~1e-13.
"""
from __future__ import annotations

import math

import numpy as np

from .evaluator import Ct, Evaluator


# ---------------------------------------------------------------------------
# slot-space linear algebra (host, float64 / complex128)

def special_fft_stages(n: int):
    """Butterfly stages S_1..S_log2(n) with V R^-1 = S_log2(n) ... S_1, as diagonal
    dictionaries {offset mod n: vector}: (S x)_a = sum_d S_d[a] x_{a+d}."""
    M = 4 * n
    rot = np.array([pow(5, j, M) for j in range(n)], dtype=np.int64)
    ksi = np.exp(2j * np.pi * np.arange(M) / M)
    a = np.arange(n)
    stages = []
    ln = 2
    while ln <= n:
        h = ln // 2
        j = a % ln
        lower = j < h
        jj = np.where(lower, j, j - h)
        t = ksi[(rot[jj] % (4 * ln)) * (M // (4 * ln))]
        stages.append(_diag_dict(n, [(0, np.where(lower, 1.0 + 0j, -t)), (h, np.where(lower, t, 0j)),
                                     (-h, np.where(lower, 0j, 1.0 + 0j))]))
        ln *= 2
    return stages


def _diag_dict(n: int, items):
    """Diagonal dictionary keyed by offset mod n; offsets that coincide mod n
    (+n/2 and -n/2) are summed."""
    out = {}
    for d, v in items:
        k = d % n
        out[k] = out[k] + v if k in out else v
    return out


def butterfly_twiddles(n: int, h: int) -> np.ndarray:
    """t_a of the stage with half-width h (defined on the lower half of each block)."""
    M = 4 * n
    ln = 2 * h
    rot = np.array([pow(5, j, M) for j in range(n)], dtype=np.int64)
    ksi = np.exp(2j * np.pi * np.arange(M) / M)
    j = np.arange(n) % ln
    jj = np.where(j < h, j, j - h)
    return ksi[(rot[jj] % (4 * ln)) * (M // (4 * ln))]


def inverse_stage(n: int, h: int):
    """Inverse of the butterfly stage with half-width h:
    x_a = (y_a + y_{a+h}) / 2,  x_{a+h} = (y_a - y_{a+h}) / (2 t_a)."""
    a = np.arange(n)
    lower = (a % (2 * h)) < h
    inv2t = 1.0 / (2.0 * butterfly_twiddles(n, h))  # t of the block's lower partner, at every a
    return _diag_dict(n, [(0, np.where(lower, 0.5 + 0j, -inv2t)), (h, np.where(lower, 0.5 + 0j, 0j)),
                          (-h, np.where(lower, 0j, inv2t))])


def compose(P: dict, Q: dict, n: int) -> dict:
    """Diagonals of P @ Q (apply Q first): (PQ)_{d+e} += P_d * Rot_d(Q_e)."""
    out = {}
    for d, pd in P.items():
        for e, qe in Q.items():
            k = (d + e) % n
            v = pd * np.roll(qe, -d)
            out[k] = out[k] + v if k in out else v
    return {k: v for k, v in out.items() if np.abs(v).max() > 0}


def apply_diags(D: dict, x: np.ndarray) -> np.ndarray:
    return sum(v * np.roll(x, -d) for d, v in D.items())


def layer_split(logn: int):
    d1 = logn // 3
    d2 = (logn - d1) // 2
    return [d1, d2, logn - d1 - d2]


def s2c_layers(n: int):
    """Three grouped layers A, B, C with V R^-1 = C B A (A applied first)."""
    stages = special_fft_stages(n)
    logn = int(math.log2(n))
    out, i = [], 0
    for size in layer_split(logn):
        M = None
        for s in stages[i:i + size]:
            M = s if M is None else compose(s, M, n)
        out.append(M)
        i += size
    return out


def c2s_layers(n: int):
    """Three grouped layers with (V R^-1)^-1 = A^-1 B^-1 C^-1 (C^-1 applied first)."""
    stages = special_fft_stages(n)
    logn = int(math.log2(n))
    inv = [inverse_stage(n, 1 << k) for k in range(len(stages))]
    groups, i = [], 0
    for size in layer_split(logn):
        groups.append(list(range(i, i + size)))
        i += size
    out = []
    for g in reversed(groups):  # C^-1 first
        M = None
        for k in reversed(g):  # within a group the highest stage is undone first
            M = inv[k] if M is None else compose(inv[k], M, n)
        out.append(M)
    return out


# ---------------------------------------------------------------------------
# Chebyshev helpers

def cheb_interp(f, K: float, deg: int) -> np.ndarray:
    k = np.arange(deg + 1)
    nodes = np.cos(np.pi * (k + 0.5) / (deg + 1))
    return np.polynomial.chebyshev.chebfit(nodes, f(K * nodes), deg)


def cheb_divide(c, m: int):
    """p = q * T_m + r for Chebyshev coefficients c (deg < 2m)."""
    c = list(c)
    d = len(c) - 1
    q = [c[m]] + [2.0 * c[m + j] for j in range(1, d - m + 1)]
    r = c[:m]
    for j in range(1, d - m + 1):
        r[m - j] -= c[m + j]
    return q, r


# ---------------------------------------------------------------------------

class LinearTransform:
    """sum_d D_d * Rot_d(x) at one level, by baby-step giant-step."""

    def __init__(self, ev: Evaluator, diags: dict, level: int, g1: int | None = None):
        self.ev, self.level = ev, level
        be = ev.be
        n = be.n // 2
        offs = sorted(diags)
        b = 0
        for d in offs:
            b = math.gcd(b, d)
        b = b or 1
        span = n // b
        ts = {}
        for d in offs:
            t = d // b
            if t > span // 2:
                t -= span
            ts[t] = diags[d]
        self.b = b
        if g1 is None:
            g1 = 1 << math.ceil(math.log2(math.sqrt(len(ts))))
        self.g1 = g1
        q = float(be.primes[level - 1])
        self.pt_scale = q
        self.groups = {}  # u -> list of (v, plaintext)
        for t, D in sorted(ts.items()):
            u, v = t // g1, t % g1
            P = np.roll(D, g1 * u * b)  # Rot_{-g1 u b}(D)
            self.groups.setdefault(u, []).append((v, ev.encode_ntt(P, q, level)))
        self.baby = sorted({v for lst in self.groups.values() for v, _ in lst})

    def steps(self):
        s = {v * self.b for v in self.baby if v}
        s |= {self.g1 * u * self.b for u in self.groups if u}
        return s

    def apply(self, x: Ct, rescale: bool = True) -> Ct:
        """With rescale=False the accumulator is returned at scale x.scale * q, one prime
        above the rescaled result, so that key switches applied to it next add noise
        divided by q (as the giant steps here do)."""
        ev, be = self.ev, self.ev.be
        if x.level != self.level:
            x = ev.drop(x, self.level)
        hoisted = ev.rotate_many(x, [v * self.b for v in self.baby if v])
        rot = {v: (x if v == 0 else hoisted[v * self.b]) for v in self.baby}
        acc = None
        for u, lst in sorted(self.groups.items()):
            inner = be.mul_plain_acc([rot[v].data for v, _ in lst], [p for _, p in lst])
            inner = x.like(inner, x.scale * self.pt_scale)
            if u:
                inner = ev.rotate(inner, self.g1 * u * self.b)
            acc = inner if acc is None else ev.add(acc, inner)
        return ev.rescale(acc) if rescale else acc


class Bootstrapper:
    def __init__(self, ev: Evaluator, scale: float = 2.0 ** 46, input_level: int = 4, K: int = 25,
                 degree: int = 47, double_angles: int = 3, F: float = 1.0 / 16):
        be = ev.be
        self.ev, self.scale, self.input_level = ev, scale, input_level
        self.K, self.r, self.F = K, double_angles, F
        self.n_slots = be.n // 2
        nq = be.nq
        self.q0 = float(be.primes[0])
        n = self.n_slots
        # SlotToCoeff at the input level; F on its last layer
        A, B, C = s2c_layers(n)
        C = {d: v * F for d, v in C.items()}
        self.s2c = [LinearTransform(ev, M, input_level - i) for i, M in enumerate((A, B, C))]
        # CoeffToSlot at the top level; 1/(2K) on its first layer
        Ci, Bi, Ai = c2s_layers(n)
        Ci = {d: v / (2.0 * K) for d, v in Ci.items()}
        self.c2s = [LinearTransform(ev, M, nq - i) for i, M in enumerate((Ci, Bi, Ai))]
        self.top = nq
        # EvalMod polynomial: cos(2 pi (K x - 1/4) / 2^r) on x in [-1, 1]
        r = double_angles
        self.cheb = cheb_interp(lambda t: np.cos(2 * np.pi * (t - 0.25) / 2 ** r), K, degree)
        self.c_fin = self.q0 / (2 * np.pi * scale * F)

    def rotation_steps(self):
        s = set()
        for lt in self.s2c + self.c2s:
            s |= lt.steps()
        return sorted(s)

    def galois_elts(self):
        ev = self.ev
        return sorted({ev.galois_elt(st) for st in self.rotation_steps()} | {2 * ev.be.n - 1})

    # ---------------- Chebyshev evaluation ----------------
    def _basis(self, x: Ct, deg: int):
        ev = self.ev
        T = {1: x}

        def prod(a, b):
            p = ev.mul_int(ev.mul(T[a], T[b]), 2)
            if a == b:
                return ev.add_const(p, -1.0)
            return ev.sub(p, ev.adjust(T[a - b], p.level, p.scale))

        g = 8
        for k in range(2, g + 1):
            if k > deg:
                break
            if k % 2 == 0:
                T[k] = prod(k // 2, k // 2)
            else:
                a = 1 << (k.bit_length() - 1)
                T[k] = prod(a, k - a)
        m = 2 * g
        while m <= deg:
            T[m] = prod(m // 2, m // 2)
            m *= 2
        return T

    def _feasible(self, T, ncoef: int, lvl: int) -> bool:
        g = 8
        d = ncoef - 1
        if d < g:
            return all(T[i].level >= lvl + 1 for i in range(1, d + 1))
        m = 1 << (d.bit_length() - 1)
        q_len = d - m + 1
        return (T[m].level >= lvl + 1 and self._feasible(T, q_len, lvl + 1) and self._feasible(T, m, lvl))

    def _eval(self, T, c, S: float, lvl: int) -> Ct:
        ev = self.ev
        d = len(c) - 1
        if d < 8:
            q = float(ev.primes[lvl])
            acc = None
            for i in range(1, d + 1):
                Ti = ev.drop(T[i], lvl + 1)
                term = ev.mul_const_unscaled(Ti, c[i], S * q / Ti.scale)
                term.scale = S * q
                acc = term if acc is None else ev.add(acc, term)
            acc = ev.add_const(acc, c[0])
            out = ev.rescale(acc)
            out.scale = S
            return out
        m = 1 << (d.bit_length() - 1)
        qc, rc = cheb_divide(c, m)
        Tm = ev.drop(T[m], lvl + 1)
        Sq = S * float(ev.primes[lvl]) / Tm.scale
        qct = self._eval(T, qc, Sq, lvl + 1)
        prod = ev.mul(qct, Tm)
        prod.scale = S
        return ev.add(prod, self._eval(T, rc, S, lvl))

    def evalmod(self, x: Ct) -> Ct:
        """x holds t / K; returns c_fin * sin(2 pi t) at scale Delta."""
        ev = self.ev
        deg = len(self.cheb) - 1
        T = self._basis(x, deg)
        lvl = x.level - 1
        while not self._feasible(T, deg + 1, lvl):
            lvl -= 1
        # backward scale targets: the i-th double angle squares at level lvl - i and drops
        # prime lvl - 1 - i, so s_in = sqrt(s_out * q); the last output scale is Delta * c_fin,
        # which reads as the value c_fin * y at scale Delta
        s = self.scale * self.c_fin
        for i in reversed(range(self.r)):
            s = math.sqrt(s * float(ev.primes[lvl - 1 - i]))
        y = self._eval(T, list(self.cheb), s, lvl)
        for _ in range(self.r):
            y = ev.add_const(ev.mul_int(ev.square(y), 2), -1.0)
        return Ct(y.data, y.scale / self.c_fin)

    # ---------------- pipeline ----------------
    def _slots_to_re_im(self, x: Ct):
        """SlotToCoeff, modraise, CoeffToSlot and the conjugation split: returns the
        real and imaginary parts (t / K) of the raised slots, same kind as x, NOT yet
        rescaled.  The last CoeffToSlot layer stops before its rescale, so the
        conjugation (and, for shared-a groups, the backward format switch) runs at
        scale q0 * q: the low-frequency part of a key switch's noise (its uncorrected
        ModUp digits are not centred) lands at the slots next to slot 0, and EvalMod
        multiplies input errors by about 2 pi K c_fin, so at scale q0 alone one
        key switch there costs ~1e-4 of output precision in those slots."""
        ev, be = self.ev, self.ev.be
        if x.level != self.input_level:
            raise ValueError(f"bootstrap input must have {self.input_level} primes")
        for lt in self.s2c:
            x = lt.apply(x)
        w = x.like(be.modraise(x.data, self.top), self.q0)
        for lt in self.c2s[:-1]:
            w = lt.apply(w)
        w = self.c2s[-1].apply(w, rescale=False)
        wc = ev.conjugate(w)
        return ev.add(w, wc), ev.mul_i(ev.sub(w, wc), sign=-1)

    def _finish(self, re: Ct, im: Ct) -> Ct:
        """Rescale the parts, EvalMod on both at once, recombine re + i im."""
        ev, be = self.ev, self.ev.be
        y = self.evalmod(ev.rescale(Ct(be.cat([re.data, im.data]), re.scale)))
        nb = re.batch
        return ev.add(Ct(y.data[:nb], y.scale), ev.mul_i(Ct(y.data[nb:], y.scale)))

    def bootstrap(self, ct: Ct) -> Ct:
        return self._finish(*self._slots_to_re_im(ct))

    def bootstrap_shared(self, ct: Ct, n: int) -> Ct:
        """Shared-a S2C-first bootstrapping of groups of n consecutive ciphertexts
        (bootstrap_shared_a_s2c_first, BatchBootstrap.cuh:719-819): FmtSwitch forward at
        the input level, SlotToCoeff / modraise / CoeffToSlot / conjugation on the
        shared-a groups with Sh-Rots, FmtSwitch backward of the real and imaginary
        parts, then EvalMod on ordinary ciphertexts."""
        ev = self.ev
        re, im = self._slots_to_re_im(ev.to_shared(ct, n))
        return self._finish(ev.from_shared(re), ev.from_shared(im))
