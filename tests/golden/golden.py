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


def c_round(x: np.ndarray) -> np.ndarray:
    """C's round(): halves away from zero."""
    return np.sign(x) * np.floor(np.abs(x) + 0.5)
