"""One BERT encoder layer through the host library (shm_boot_bert_layer; the reference's
src/include/test/test_single_layer.cuh:422-2062 with single_att_block.cuh:21-315), at reduced
width on N = 2^12 with the reference's layer chain (35 + 5 primes): 64 inputs x 32 tokens fill
the 2,048 slots, hidden 16 in 2 heads, FFN 64.  The decrypted output is compared with
the FP64 layer that uses the same approximations (shmoai_b200/plain_layer.py, approx: the
encryption's own error) and with the exact FP64 layer.  CPU: the oracle build, shared-a form.
GPU: the CUDA build equals the oracle build bit for bit, and the per-ciphertext ("orig") form
agrees with the shared-a ("sham") form within the bootstrap's error."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from shmoai_b200 import plain_layer as P
from shmoai_b200.host import BERT_STAGES, Bootstrapper, Host

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_HOST = os.path.join(ROOT, "oracle", "_build", "libshmoai_host_oracle.so")
# the reference's layer chain for the shared-a form (test_single_layer.cuh:503-530): three 46-bit primes
# where the bootstrap region starts, so every rescale after a bootstrap (at 23 primes) is by a 46-bit prime
LAYER_BITS = [51] + [46] * 23 + [51] * 11 + [51] * 5
CFG = dict(hidden=16, heads=2, ffn=64, num_X=64, tokens=32, input_num=32, softmax_iter=13, ln_newt=3,
           ln_gold=2, gelu_input_level=13, ffn_chunk=32, members=2, boot_batch=16, w_scale=2.0 ** 40,
           ln_var_scale=64.0)


def _run(lib, members, boot_batch):
    cfg = dict(CFG, members=members, boot_batch=boot_batch)
    h = Host(12, O.gen_primes(12, LAYER_BITS), 5, hamming_weight=64, seed=31, lib=lib)
    h.gen_relin_key()
    h.gen_public_key(5)
    bs = Bootstrapper(h, 2.0 ** 46, 4)
    nb = (h.n // 2) // cfg["tokens"]
    ct_elts = [h.galois_elt(i * nb) for i in range(1, cfg["tokens"])]
    if members:  # the attention's rotation keys are made inside the layer call and released after it
        h.gen_shared_keys(members, bs.galois_elts(), hamming_weight=64)
    else:
        h.gen_galois_keys(sorted(set(bs.galois_elts()) | set(ct_elts)))
    rng = np.random.default_rng(77)
    X = rng.normal(0, 1, (cfg["num_X"], cfg["tokens"], cfg["hidden"]))
    w = P.random_weights(rng, cfg["hidden"], cfg["ffn"])
    mask = np.ones(h.n // 2, dtype=np.int32)
    ct = h.batch_input(X, 2.0 ** 46, 23)
    out, times = bs.bert_layer(ct, w, cfg, mask)
    assert list(times) == BERT_STAGES and all(t >= 0 for t in times.values())
    assert (out.count, out.level) == (cfg["hidden"], 23) and abs(out.scale / 2.0 ** 46 - 1) < 1e-12
    got = h.decrypt(out).real
    cols = P.pack_columns(X)
    approx = P.layer(cols, w, cfg, mask, approx=True)
    exact = P.layer(cols, w, cfg, mask, approx=False)
    return out.to_host(), got, approx, exact


def test_layer_on_oracle_matches_fp64_layer():
    _, got, approx, exact = _run(ORACLE_HOST, 2, 16)
    e_approx = np.abs(got - approx)
    e_exact = np.abs(got - exact)
    # the encryption's own error (bootstraps, rescales) after two LayerNorms' amplification
    assert e_approx.mean() < 2e-4 and e_approx.max() < 5e-3, (e_approx.mean(), e_approx.max())
    # plus the approximations' error (exp, inverse, 1/sqrt, the GELU series)
    assert e_exact.mean() < 2e-2 and e_exact.max() < 5e-2, (e_exact.mean(), e_exact.max())


@pytest.mark.gpu
def test_layer_cuda_matches_oracle_build_and_orig_form():
    words, got, approx, _ = _run(None, 2, 16)
    words_o, _, _, _ = _run(ORACLE_HOST, 2, 16)
    assert np.array_equal(words, words_o)
    _, got_orig, _, _ = _run(None, 0, 1)
    assert np.abs(got_orig - approx).mean() < 2e-4 and np.abs(got_orig - approx).max() < 5e-3
    assert np.abs(got_orig - got).max() < 5e-3
