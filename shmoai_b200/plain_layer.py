"""The BERT encoder layer in FP64 on plaintext slot vectors: the model that the encrypted layer
(shm_boot_bert_layer) is measured against.

Layout: the MOAI column packing (Batch_encode_encrypt.cuh:12-43) - one slot vector per hidden
column, slot num_X * t + s holding token t of input s.  Two forms:

  exact   the layer itself: softmax with exp and a true division, LayerNorm with 1/sqrt, GELU by
          erf (the FP64 plaintext layer that the encrypted output's error is quoted against);
  approx  the same layer with the encrypted pipeline's approximations in FP64: exp by
          (1 + x/128)^128 after a shift of -8.1, the softmax sum's inverse by the product
          prod_i (1 + y^(2^i)), LayerNorm's 1/sqrt by the linear guess, Newton and Goldschmidt
          steps on var_scale * var, GELU by the reference's degree-24 Chebyshev series on
          [-19.5, 12.5] (src/include/source/non_linear_func/: softmax.cuh:23-118,
          layernorm.cuh:708-897, gelu_other.cuh:258-300).  The difference between the encrypted
          output and this form is the encryption's own error.
"""
from __future__ import annotations

import math

import numpy as np

# gelu_cheb's coefficients (gelu_other.cuh:284-296), the same series the encrypted GELU evaluates
GELU_SERIES = np.array([
    3.4550752799e+00, 5.7852067632e+00, 3.1727714170e+00, 7.0234932500e-01, -4.6200569546e-01,
    -3.7817535966e-01, 8.4136420694e-02, 2.2427456987e-01, 2.9451916291e-02, -1.2928072669e-01,
    -6.6659430283e-02, 6.4349502364e-02, 7.1733295078e-02, -1.9882581810e-02, -6.1145844240e-02,
    -8.4827295421e-03, 4.3597254356e-02, 2.3373027950e-02, -2.4790187963e-02, -2.7940100474e-02,
    8.8404026343e-03, 2.3776567058e-02, 8.8171887083e-03, -4.6290425955e-02, -9.7997267900e-03])
GELU_LO, GELU_HI = -19.5, 12.5
SOFTMAX_SHIFT = -8.1


def pack_columns(X: np.ndarray) -> np.ndarray:
    """[num_X][tokens][hidden] -> [hidden][slots] with slot num_X * t + s."""
    nx, nt, d = X.shape
    return np.ascontiguousarray(X.transpose(2, 1, 0).reshape(d, nt * nx))


def unpack_columns(cols: np.ndarray, num_X: int) -> np.ndarray:
    d, slots = cols.shape
    return cols.reshape(d, slots // num_X, num_X).transpose(2, 1, 0)


def gelu_exact(x):
    try:
        from scipy.special import erf
    except ImportError:  # element by element (slow at full width)
        erf = np.vectorize(math.erf)
    return 0.5 * x * (1.0 + erf(x / math.sqrt(2.0)))


def gelu_approx(x):
    return np.polynomial.chebyshev.chebval((2 * x - GELU_HI - GELU_LO) / (GELU_HI - GELU_LO), GELU_SERIES)


def exp_approx(y):
    return (1.0 + y / 128.0) ** 128


def inverse_approx(x, iters: int):
    y = 1.0 - x
    r = 1.0 + y
    for _ in range(iters):
        y = y * y
        r = r * (1.0 + y)
    return r


def inv_sqrt_approx(x, newt: int, gold: int):
    r = -1.29054537e-4 * x + 0.129054537
    for _ in range(newt):
        r = r * (1.5 - 0.5 * x * r * r)
    g, h = x * r, 0.5 * r
    for _ in range(gold):
        s = 0.5 - g * h
        g, h = g + g * s, h + h * s
    return 2.0 * h


def _layernorm(x, gamma, beta, approx: bool, cfg: dict):
    mean = x.mean(axis=0, keepdims=True)
    xc = x - mean
    var = (xc * xc).mean(axis=0, keepdims=True)
    if approx:
        c = cfg.get("ln_var_scale", 64.0)
        inv = inv_sqrt_approx(c * var, cfg["ln_newt"], cfg["ln_gold"]) * math.sqrt(c)
    else:
        inv = 1.0 / np.sqrt(var)
    return gamma[:, None] * xc * inv + beta[:, None]


def layer(cols: np.ndarray, w: dict, cfg: dict, mask: np.ndarray, approx: bool) -> np.ndarray:
    """One layer on [hidden][slots] FP64 columns; w as in Bootstrapper.bert_layer; mask the bias_vec
    slots (full rows: every key of a query row is valid)."""
    d, F, H = cfg["hidden"], cfg["ffn"], cfg["heads"]
    nx, nt = cfg["num_X"], cfg["tokens"]
    dh = d // H
    m = mask.astype(np.float64)[None, :]
    Q = (w["Wq"].T @ cols + w["bq"][:, None] * m) / math.sqrt(dh)
    K = w["Wk"].T @ cols + w["bk"][:, None] * m
    V = w["Wv"].T @ cols + w["bv"][:, None] * m
    heads = []
    for h in range(H):
        sl = slice(h * dh, (h + 1) * dh)
        q = Q[sl].reshape(dh, nt, nx)
        k = K[sl].reshape(dh, nt, nx)
        v = V[sl].reshape(dh, nt, nx)
        s = np.einsum("jts,jus->stu", q, k)  # [input][query token][key token]
        if approx:
            e = exp_approx(s + SOFTMAX_SHIFT)
            p = e * inverse_approx(e.sum(axis=2, keepdims=True), cfg["softmax_iter"])
        else:
            e = np.exp(s - s.max(axis=2, keepdims=True))
            p = e / e.sum(axis=2, keepdims=True)
        heads.append(np.einsum("stu,jus->jts", p, v).reshape(dh, nt * nx))
    att = np.concatenate(heads)
    S = w["Wo"].T @ att + w["bo"][:, None] * m
    H1 = _layernorm(S + cols, w["ln1_gamma"], w["ln1_beta"], approx, cfg)
    I = w["Wi"].T @ H1 + w["bi"][:, None] * m
    G = gelu_approx(I) if approx else gelu_exact(I)
    Fo = (w["Wf"].T @ G) * m + w["bf"][:, None] * m
    return _layernorm(Fo + H1, w["ln2_gamma"], w["ln2_beta"], approx, cfg)


def random_weights(rng: np.random.Generator, d: int, F: int, std: float = 0.02) -> dict:
    """Random-init weights N(0, std^2); LayerNorm gamma 1 and beta 0 (BERT's initialisation)."""
    def n(*shape):
        return rng.normal(0.0, std, shape)

    return {"Wq": n(d, d), "bq": n(d), "Wk": n(d, d), "bk": n(d), "Wv": n(d, d), "bv": n(d), "Wo": n(d, d),
            "bo": n(d), "ln1_gamma": np.ones(d), "ln1_beta": np.zeros(d), "Wi": n(d, F), "bi": n(F),
            "Wf": n(F, d), "bf": n(d), "ln2_gamma": np.ones(d), "ln2_beta": np.zeros(d)}
