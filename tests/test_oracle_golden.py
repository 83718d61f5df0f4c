"""The CPU oracle against the reference's own outputs (golden fixtures made by
running the reference evaluator built for sm_100a, tests/golden/make_golden.py).

Every record is checked bit for bit (checksum over all limbs + the first 8
coefficients of each limb)."""
import numpy as np
import pytest

from golden.golden import GoldenSet, c_round
from oracle import oracle as O

SETS = ["tiny", "prim", "boot"]
OPS = ["intt_A", "ntt_A", "add_AB", "mulplain_AC", "rescale_A", "rot1_A", "conj_A", "mul_AB", "relin_AB",
       "mrr_AB", "rot1_D", "relin_DE"]


@pytest.fixture(scope="module", params=SETS)
def computed(request):
    g = GoldenSet(request.param)
    o = O.Oracle(g.log_n, g.primes, g.nq, g.np)
    A, B, C = g.ct(1), g.ct(2), g.plain(3)
    rk, gk5, gkc = g.relin_key(), g.galois_key(5), g.galois_key(2 * g.n - 1)
    r = {"intt_A": o.intt(A), "ntt_A": o.ntt(A), "add_AB": o.add(A, B), "mulplain_AC": o.multiply_plain(A, C),
         "rescale_A": o.rescale(A), "rot1_A": o.apply_galois_ct(A, 5, gk5),
         "conj_A": o.apply_galois_ct(A, 2 * g.n - 1, gkc)}
    m = o.tensor(A, B)
    r["mul_AB"] = m
    r["relin_AB"] = o.relinearize(m, rk)
    r["mrr_AB"] = o.rescale(r["relin_AB"])
    D, E = g.ct(4, g.L - 1), g.ct(5, g.L - 1)
    r["rot1_D"] = o.apply_galois_ct(D, 5, gk5)
    r["relin_DE"] = o.relinearize(o.tensor(D, E), rk)
    W, X = g.ctpt_weights(), g.ctpt_inputs()
    Y = o.ctpt_matmul(X, W)
    for k in range(W.shape[1]):
        r[f"ctpt_sum_{k}"] = Y[k]
        r[f"ctpt_out_{k}"] = o.rescale(np.ascontiguousarray(Y[k]))
    return g, o, r


def test_params_match_reference_primes(computed):
    g, o, _ = computed
    log_n, bits, np_ = O.PARAM_SETS[g.name]
    assert np.array_equal(O.gen_primes(log_n, bits), g.primes)
    assert (g.nq, g.np) == (len(bits) - np_, np_)


@pytest.mark.parametrize("op", OPS)
def test_oracle_op_bit_exact(computed, op):
    g, _, r = computed
    ok, msg = g.matches(op, r[op])
    assert ok, msg


def test_oracle_ctpt_bit_exact(computed):
    g, _, r = computed
    n_out = g.ctpt_weights().shape[1]
    for k in range(n_out):
        for name in (f"ctpt_sum_{k}", f"ctpt_out_{k}"):
            ok, msg = g.matches(name, r[name])
            assert ok, msg


def test_constant_encode_is_rounded_product(computed):
    """The reference's FP64 encode of a constant (moai::Encoder::encode(double))
    equals C round(w * 2^40) for every sampled weight, exact ties included."""
    g, _, _ = computed
    vals = g.record("encode_w")["values"]
    w = np.array([v[0] for v in vals])
    c = np.array([int(v[1]) for v in vals], dtype=np.int64)
    assert all(v[2] == 1 for v in vals), "encoded constant is not constant across slots"
    assert np.array_equal(c_round(w * 2.0 ** 40).astype(np.int64), c)


def test_ctpt_weights_are_rounded_products(computed):
    g, _, _ = computed
    W = g.ctpt_weights()
    w = np.array(g.record("ctpt_w")).reshape(W.shape)
    assert np.array_equal(c_round(w * 2.0 ** 40).astype(np.int64), W)
