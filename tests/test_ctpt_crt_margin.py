"""The tensor-core ct-pt matmul's residue system (shmoai_b200/csrc/ctpt_tc.cu: make_plan, crt_kernel),
restated with Python integers at its edge cases: a limb of prime q takes the first T moduli whose
product M satisfies log2 M >= log2 B + 1.05 with B = (q - 1) max_o sum_i |w_io|, and the fold takes
v = round(sum_t r_t frac_t) in 19-bit fixed point, F_t = round(2^19 [(M/m_t)^-1]_{m_t} / m_t),
v = (sum_t r_t F_t + 2^18) >> 19.  For every |S| <= B, S = sum_t r_t c_t - v M must hold exactly
(c_t = (M/m_t) [(M/m_t)^-1]_{m_t}), including S = +-B and the sums whose fraction lies closest to
one half.  Also checks the bench's restatement of the moduli counts against the same rule."""
import math

import numpy as np

MODULI = [251, 241, 239, 233, 229, 227, 223, 211, 199, 197, 193, 191, 181, 179, 173, 167, 163, 157, 151, 149]
FRAC_BITS = 19


def moduli_count(q, l1):
    need = math.log2(q - 1) + math.log2(max(l1, 1)) + 1.05
    have, T = 0.0, 0
    while have < need:
        have += math.log2(MODULI[T])
        T += 1
    return T


def fold(S, T):
    ms = MODULI[:T]
    M = math.prod(ms)
    r = [S % m for m in ms]  # the GEMM's residues in [0, m_t)
    acc, v_acc = 0, 1 << (FRAC_BITS - 1)
    for t, m in enumerate(ms):
        Mt = M // m
        inv = pow(Mt % m, -1, m)
        acc += r[t] * Mt * inv
        v_acc += r[t] * ((inv << FRAC_BITS) + m // 2) // m
    assert v_acc < 1 << 32  # the kernel's 32-bit sum
    v = v_acc >> FRAC_BITS
    return acc - v * M


def test_fold_exact_at_the_bound():
    rng = np.random.default_rng(5)
    for q_bits in (36, 46, 51, 60):
        q = (1 << q_bits) - 1
        for l1 in (1, 3, 768 * (1 << 36), 3072 * (1 << 39), (1 << 59) // q_bits):
            T = moduli_count(q, l1)
            if T > len(MODULI):
                continue
            B = (q - 1) * l1
            M = math.prod(MODULI[:T])
            assert M >= 2.02 * B
            cases = [B, -B, 0, 1, -1, B - 1, -(B - 1)]
            # the fractions closest to one half that |S| <= B allows: S near +-M/2.02
            cases += [int(rng.integers(-B, B, dtype=np.int64)) if B < 2 ** 62 else
                      int(rng.integers(0, 2 ** 62)) * (B >> 62) * (1 if k % 2 else -1) for k in range(40)]
            for S in cases:
                assert fold(S, T) == S, (q_bits, l1, T, S)


def test_fixed_point_error_bound():
    """sum_t r_t |F_t / 2^19 - frac_t| < 0.005 for every moduli count and residues up to m_t - 1."""
    for T in range(1, len(MODULI) + 1):
        ms = MODULI[:T]
        M = math.prod(ms)
        err = 0.0
        for m in ms:
            inv = pow((M // m) % m, -1, m)
            F = ((inv << FRAC_BITS) + m // 2) // m
            err += (m - 1) * abs(F / 2 ** FRAC_BITS - inv / m)
        assert err < 0.005, (T, err)


def test_bench_restatement_matches_rule():
    import sys
    import os

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch

    import bench
    from oracle import oracle as O

    log_n = bench.BOOT["log_n"]
    primes = [int(p) for p in O.gen_primes(log_n, bench.BOOT["bits"])]

    class Ctx:
        pass

    ctx = Ctx()
    ctx.primes = np.array(primes, dtype=np.uint64)
    ctx.n = 1 << log_n
    g = torch.Generator().manual_seed(2)
    W = torch.round(torch.randn(768, 768, generator=g, dtype=torch.float64) * 0.02 * 2 ** 40).to(torch.int64)
    l1 = int(W.abs().sum(0).max().item())
    L = 13
    counts = bench.ctpt_moduli_counts(ctx, W, L)
    limb_t = [moduli_count(primes[l], l1) for l in range(L)]
    n, R = ctx.n, 2 * L * ctx.n
    want = []
    for r0 in range(0, R, 131072):
        rows = range(r0 // n, (r0 + 131072 - 1) // n + 1)
        want.append(max(limb_t[r % L] for r in rows))
    assert [t for t, _ in counts] == want
    assert set(want) == {12, 13}  # the 46-bit limbs need 12 moduli, the 51-bit one 13
