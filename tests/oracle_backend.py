"""The CPU oracle behind the backend interface of shmoai_b200.backend.GpuBackend.

TEST INFRASTRUCTURE ONLY: lets the scale-exact evaluator and the bootstrapping
pipeline run on the CPU oracle (numpy arrays, oracle/ckks_oracle.c arithmetic)
so their host logic is checked without a GPU, at small ring degrees.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O


class OracleBackend:
    name = "oracle"

    def __init__(self, log_n: int, bits, n_special: int):
        self.o = O.Oracle.from_bits(log_n, bits, n_special)
        self.n, self.log_n = self.o.n, log_n
        self.nq, self.np, self.dnum = self.o.nq, self.o.np, self.o.dnum
        self.primes = [int(p) for p in self.o.primes]
        self._pq = np.array(self.primes, dtype=np.uint64)

    # memory
    def from_host(self, a):
        return np.ascontiguousarray(a, dtype=np.uint64)

    def to_host(self, t):
        return t

    def empty(self, *shape):
        return np.empty(shape, dtype=np.uint64)

    def stack(self, ts):
        return np.stack(list(ts))

    def cat(self, ts):
        return np.concatenate(list(ts), axis=0)

    def clone(self, t):
        return t.copy()

    def take_poly(self, t, i):
        return np.ascontiguousarray(t[:, i])

    def _q(self, L):
        return self._pq[:L].reshape(L, 1)

    # ring operations
    def ntt_fwd(self, t):
        t[...] = self.o.ntt(t)
        return t

    def ntt_inv(self, t):
        t[...] = self.o.intt(t)
        return t

    def add(self, a, b, out=None):
        q = self._q(a.shape[-2])
        s = a + b
        r = np.where(s >= q, s - q, s)
        return r

    def sub(self, a, b, out=None):
        q = self._q(a.shape[-2])
        return np.where(a >= b, a - b, a + q - b)

    def neg(self, a, out=None):
        q = self._q(a.shape[-2])
        return np.where(a == 0, a, q - a)

    def mul_plain(self, ct, pt, out=None):
        return self.o.multiply_plain(np.ascontiguousarray(ct), np.ascontiguousarray(pt))

    def tensor(self, a, b):
        return np.stack([self.o.tensor(np.ascontiguousarray(a[i]), np.ascontiguousarray(b[i]))
                         for i in range(a.shape[0])])

    def relin(self, ct3, key):
        return np.stack([self.o.relinearize(np.ascontiguousarray(c), key) for c in ct3])

    def rescale(self, t):
        return self.o.rescale(np.ascontiguousarray(t))

    def apply_galois(self, ct, elt, key):
        return np.stack([self.o.apply_galois_ct(np.ascontiguousarray(c), elt, key) for c in ct])

    def apply_galois_many(self, ct, elts, keys):
        per_ct = [self.o.apply_galois_hoisted(np.ascontiguousarray(c), elts, keys) for c in ct]
        return [np.stack([per_ct[i][e] for i in range(len(ct))]) for e in range(len(elts))]

    def sh_rotate_many(self, sh, elts, keys):
        per_g = [self.o.shared_rotate_hoisted(np.ascontiguousarray(g), elts, keys) for g in sh]
        return [np.stack([per_g[g][e] for g in range(len(sh))]) for e in range(len(elts))]

    def fmt_forward(self, cts, n, key):
        return np.stack([self.o.fmt_forward(cts[g * n:(g + 1) * n], key) for g in range(cts.shape[0] // n)])

    def fmt_backward(self, sh, keys):
        return np.concatenate([self.o.fmt_backward(np.ascontiguousarray(g), keys) for g in sh])

    def permute_plain(self, pt, elt):
        return np.ascontiguousarray(pt[..., O.galois_perm(self.log_n, elt)])

    def mul_scalar(self, a, residues, out=None):
        L = a.shape[-2]
        pt = np.repeat(np.asarray(residues[:L], dtype=np.uint64).reshape(L, 1), self.n, axis=1)
        return self.o.multiply_plain(np.ascontiguousarray(a), pt)

    def add_scalar(self, ct, residues, out=None):
        L = ct.shape[-2]
        r = ct.copy()
        c0 = r[:, 0]
        s = c0 + np.asarray(residues[:L], dtype=np.uint64).reshape(L, 1)
        q = self._q(L)
        r[:, 0] = np.where(s >= q, s - q, s)
        return r

    def mul_plain_acc(self, cts, pts, out=None, accumulate=False):
        acc = None
        for c, p in zip(cts, pts):
            t = self.mul_plain(c, p)
            acc = t if acc is None else self.add(acc, t)
        return acc

    def modraise(self, ct1, L):
        c = self.o.intt(np.ascontiguousarray(ct1))[..., 0, :]  # [n][2][N] mod q0
        q0 = self.primes[0]
        v = c.astype(np.int64)
        v = np.where(c > np.uint64(q0 // 2), v - q0, v)
        out = np.stack([np.remainder(v, np.int64(self.primes[j])).astype(np.uint64) for j in range(L)], axis=-2)
        return self.o.ntt(np.ascontiguousarray(out))

    def drop(self, t, L_out):
        return np.ascontiguousarray(t[..., :L_out, :])

    def uniform(self, shape, rows, gen):
        raise NotImplementedError

    def synchronize(self):
        pass
