"""The oracle's number theory against the reference's own host code
(oracle/_ref/libref_host.so, compiled from the reference sources)."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

R = O.ref_host()
pytestmark = pytest.mark.skipif(R is None, reason="reference host library not built (oracle/build_ref.sh)")


@pytest.mark.parametrize("name", list(O.PARAM_SETS))
def test_primes(name):
    log_n, bits, _ = O.PARAM_SETS[name]
    ref = np.zeros(len(bits), dtype=np.uint64)
    assert R.ref_create_primes(log_n, (ctypes.c_int * len(bits))(*bits), len(bits), O._p(ref)) == 0
    assert np.array_equal(O.gen_primes(log_n, bits), ref)


@pytest.mark.parametrize("name", list(O.PARAM_SETS))
def test_ntt_tables(name):
    log_n, bits, _ = O.PARAM_SETS[name]
    primes = O.gen_primes(log_n, bits)
    n = 1 << log_n
    for q in [int(primes[0]), int(primes[1]), int(primes[-1])]:
        rp, irp = O.ntt_tables(q, log_n)
        rrp, rirp = np.zeros(n, np.uint64), np.zeros(n, np.uint64)
        root, ninv = np.zeros(1, np.uint64), np.zeros(1, np.uint64)
        assert R.ref_ntt_tables(log_n, q, O._p(rrp), O._p(rirp), O._p(root), O._p(ninv)) == 0
        assert int(root[0]) == int(rp[1 << (log_n - 1)])  # psi^1 sits at bitrev(1)
        assert np.array_equal(rp, rrp)
        folded = irp.copy()
        folded[1] = (int(irp[1]) * int(ninv[0])) % q  # the reference folds N^-1 into entry 1
        assert np.array_equal(folded, rirp)


def test_base_converter_constants():
    log_n, bits, np_ = O.PARAM_SETS["boot"]
    pr = [int(x) for x in O.gen_primes(log_n, bits)]
    ib, ob = pr[:5], pr[5:12]
    qhi, qhm = np.zeros(5, np.uint64), np.zeros(7 * 5, np.uint64)
    assert R.ref_base_converter(O._p(np.array(ib, np.uint64)), 5, O._p(np.array(ob, np.uint64)), 7, O._p(qhi),
                                O._p(qhm)) == 0
    for i in range(5):
        h = 1
        for k in range(5):
            if k != i:
                h *= ib[k]
        assert pow(h % ib[i], -1, ib[i]) == int(qhi[i])
        for j in range(7):
            assert h % ob[j] == int(qhm[j * 5 + i])
