"""Key generation, encryption and decryption for the scale-exact evaluator.

Follows the reference's key structure (thirdparty/phantom-fhe/src/secretkey.cu):
  * secret s: ternary with exactly h non-zero coefficients (gen_secretkey +
    the MOAI Hamming-weight trim, secretkey.cu:376-522);
  * errors: centred binomial over 21 + 21 bits, sigma ~ 3.24 (src/prng.cu:217-240);
  * key-switching key for s' (generate_one_kswitch_key, secretkey.cu:328-373):
    dnum digits, digit b = [ -(a_b s + e_b) + P * [digit-b CRT unit] * s',  a_b ]
    over the whole QP basis, laid out [dnum][2][QP][N];
  * relinearisation key: s' = s^2; Galois key of element g: s' = sigma_g(s).
Encryption here is symmetric (c0 = -(a s) + e + m, c1 = a); the reference's
public-key encryption (secretkey.cu:15-217) gives ciphertexts of the same form
with a slightly larger fresh error.

Sampling uses numpy / torch generators seeded by the caller; this is setup work
and is not on the timed path.
"""
from __future__ import annotations

import numpy as np

from .encoder import Encoder
from .evaluator import Ct


def cbd(rng: np.random.Generator, shape) -> np.ndarray:
    mask = np.uint64((1 << 21) - 1)
    a = rng.integers(0, 2 ** 63, size=shape, dtype=np.uint64) & mask
    b = rng.integers(0, 2 ** 63, size=shape, dtype=np.uint64) & mask
    return np.bitwise_count(a).astype(np.int64) - np.bitwise_count(b).astype(np.int64)


class KeyGenerator:
    def __init__(self, backend, hamming_weight: int = 192, seed: int = 0x5EED):
        import torch

        self.be = backend
        self.n = backend.n
        self.QP = backend.nq + backend.np
        self.rng = np.random.default_rng(seed)
        self.tgen = torch.Generator(device="cuda").manual_seed(seed) if backend.name == "cuda" else None
        self.enc = Encoder(backend.log_n)
        s = np.zeros(self.n, dtype=np.int64)
        pos = self.rng.choice(self.n, size=hamming_weight, replace=False)
        s[pos] = self.rng.choice(np.array([-1, 1], dtype=np.int64), size=hamming_weight)
        self.s_coeffs = s
        self.s = self._ntt_qp(s)  # [QP][N]

    # ---------------- helpers ----------------
    def _ntt_qp(self, coeffs) -> object:
        t = self.be.from_host(self.enc.to_rns(coeffs, self.be.primes))
        return self.be.ntt_fwd(t)

    def _uniform(self, shape):
        """Uniform residues, last-but-one axis over the first shape[-2] primes."""
        L = shape[-2]
        if self.be.name == "cuda":
            return self.be.uniform(shape, list(range(L)), self.tgen)
        out = np.empty(shape, dtype=np.uint64)
        for i in range(L):
            out[..., i, :] = self.rng.integers(0, self.be.primes[i], size=shape[:-2] + (shape[-1],),
                                               dtype=np.uint64)
        return self.be.from_host(out)

    def _error_ntt(self, lead, L):
        e = cbd(self.rng, tuple(lead) + (self.n,))
        rns = np.stack([np.remainder(e, np.int64(q)).astype(np.uint64) for q in self.be.primes[:L]], axis=-2)
        return self.be.ntt_fwd(self.be.from_host(rns))

    # ---------------- keys ----------------
    def switching_key(self, s_new):
        """[dnum][2][QP][N] key switching s_new -> s."""
        be, QP, np_, nq = self.be, self.QP, self.be.np, self.be.nq
        P = 1
        for p in be.primes[nq:]:
            P *= p
        digits = []
        for b in range(be.dnum):
            a = self._uniform((1, QP, self.n))
            e = self._error_ntt((1,), QP)
            bpart = be.sub(e, be.mul_plain(a, self.s))  # e - a s
            unit = np.zeros(QP, dtype=np.uint64)
            for i in range(b * np_, min((b + 1) * np_, nq)):
                unit[i] = P % be.primes[i]
            bpart = be.add(bpart, be.mul_scalar(self._as_poly(s_new), unit))
            digits.append(be.stack([bpart[0], a[0]]))
        return be.stack(digits)

    def _as_poly(self, t):
        return t.reshape((1,) + tuple(t.shape)) if hasattr(t, "reshape") else t[None]

    def relin_key(self):
        s2 = self.be.mul_plain(self._as_poly(self.s), self.s)[0]
        return self.switching_key(s2)

    def galois_key(self, elt: int):
        return self.switching_key(self.be.permute_plain(self.s, elt))

    # ---------------- shared-a keys ----------------
    def aux_secrets(self, n: int, hamming_weight: int = 192):
        """n auxiliary secrets s'_i of a shared-a group (SharedAKeyGen, FmtSwitch.cuh:235-305),
        ternary with exactly `hamming_weight` non-zero coefficients, NTT form over QP."""
        out = []
        for _ in range(n):
            s = np.zeros(self.n, dtype=np.int64)
            pos = self.rng.choice(self.n, size=hamming_weight, replace=False)
            s[pos] = self.rng.choice(np.array([-1, 1], dtype=np.int64), size=hamming_weight)
            out.append(self._ntt_qp(s))
        self.aux = out
        return out

    def _p_units(self, digit: int | None):
        """Residues of P * E_digit over QP (E the CRT unit of the digit's primes), or of P
        on every Q prime when digit is None."""
        be, nq = self.be, self.be.nq
        P = 1
        for p in be.primes[nq:]:
            P *= p
        unit = np.zeros(self.QP, dtype=np.uint64)
        rows = range(nq) if digit is None else range(digit * be.np, min((digit + 1) * be.np, nq))
        for i in rows:
            unit[i] = P % be.primes[i]
        return unit

    def _multi_key(self, olds, adds):
        """[D][n + 1][QP][N]: digit d = (B_{d,0} .. B_{d,n-1}, A_d) with
        B_{d,i} = e_{d,i} - A_d * olds[i] (+ unit * s_new for each (i, unit, s_new) in adds[d])."""
        be = self.be
        digits = []
        for add in adds:
            A = self._uniform((1, self.QP, self.n))
            rows = []
            for so in olds:
                e = self._error_ntt((1,), self.QP)
                rows.append(be.sub(e, be.mul_plain(A, so)))
            for i, unit, sn in add:
                rows[i] = be.add(rows[i], be.mul_scalar(self._as_poly(sn), unit))
            rows.append(A)
            digits.append(be.cat(rows))
        return be.stack(digits)

    def shared_galois_key(self, elt: int):
        """Sh-Galois key of element g (gen_shared_galois_key, ShRotate.cu:54-162):
        [dnum][n + 1][QP][N], B_{d,i} = -A_d s'_i + e + P E_d sigma_g(s'_i), one A_d per digit."""
        news = [self.be.permute_plain(s, elt) for s in self.aux]
        adds = [[(i, self._p_units(d), news[i]) for i in range(len(self.aux))] for d in range(self.be.dnum)]
        return self._multi_key(self.aux, adds)

    def format_key(self):
        """FmtSwitch forward key (gen_format_key, FmtSwitch.cu:165-270): [n][n + 1][QP][N],
        digit j = member j's a; B_fmt[j][i] = -a_fmt[j] s'_i + e + [i == j] P s."""
        n = len(self.aux)
        unit = self._p_units(None)
        return self._multi_key(self.aux, [[(j, unit, self.s)] for j in range(n)])

    def backward_keys(self):
        """FmtSwitch backward keys: the switching key s'_i -> s of every member."""
        return [self.switching_key(s) for s in self.aux]

    def decrypt_shared_coeffs(self, sh) -> np.ndarray:
        """Centred coefficients [G * n][N] of shared-a groups [G][n + 1][L][N] (b_i + a s'_i)."""
        be = self.be
        d = be.drop(sh, 1) if sh.shape[-2] > 1 else sh
        n = d.shape[1] - 1
        out = []
        for g in range(d.shape[0]):
            grp = d[g]
            for i in range(n):
                m = be.add(grp[i:i + 1], be.mul_plain(grp[n:n + 1], self.aux[i][:1]))
                m = be.ntt_inv(be.clone(m))
                out.append(self.enc.centered(be.to_host(m)[:, 0, :], be.primes[0])[0])
        return np.stack(out)

    def decrypt_shared(self, sh, scale: float) -> np.ndarray:
        return np.stack([self.enc.decode(c, scale) for c in self.decrypt_shared_coeffs(sh)])

    # ---------------- encryption ----------------
    def encrypt(self, z_batch, scale: float, L: int) -> Ct:
        """Encrypt each row of z_batch (complex slot vectors) at level L and `scale`."""
        be = self.be
        ms = [self.enc.to_rns(self.enc.encode(z, scale), be.primes[:L]) for z in z_batch]
        m = be.ntt_fwd(be.from_host(np.stack(ms)))  # [n][L][N]
        n = len(ms)
        a = self._uniform((n, L, self.n))
        e = self._error_ntt((n,), L)
        s_L = self.s[:L]
        c0 = be.add(be.sub(e, be.mul_plain(a, s_L)), m)
        data = be.stack([be.stack([c0[i], a[i]]) for i in range(n)])
        return Ct(data, scale)

    def decrypt_coeffs(self, ct: Ct) -> np.ndarray:
        """Centred plaintext coefficients (float64, [n][N]) via the first limb
        (exact while |m| < q0 / 2)."""
        be = self.be
        d = be.drop(ct.data, 1) if ct.level > 1 else ct.data
        s1 = self.s[:1]
        c0, c1 = be.take_poly(d, 0), be.take_poly(d, 1)
        m = be.add(c0, be.mul_plain(c1, s1))
        m = be.ntt_inv(be.clone(m))
        return self.enc.centered(be.to_host(m)[:, 0, :], be.primes[0])

    def decrypt(self, ct: Ct) -> np.ndarray:
        """Complex slot values [n][N/2]."""
        return np.stack([self.enc.decode(c, ct.scale) for c in self.decrypt_coeffs(ct)])
