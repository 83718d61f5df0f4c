/*
 * CPU oracle for the RNS-CKKS evaluator hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is loaded by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and
 * never by the product library (shmoai_b200/), which has its own host math
 * and CUDA kernels.
 *
 * It restates, in plain scalar C (OpenMP over limbs), the arithmetic of the
 * reference evaluator (ShMOAI's vendored PhantomFHE):
 *
 *   prime chain        thirdparty/phantom-fhe/src/modulus.cu:79-110 (CoeffModulus::Create,
 *                      per-bit-size lists assigned from the back) and
 *                      src/util/numth.cu:209-235 (get_primes: 2^b - 2N + 1 downwards)
 *   NTT tables         src/util/ntt.cu:11-56 (minimal primitive 2N-th root,
 *                      root_powers[bitrev(i)] = psi^i)
 *   forward / inverse  src/ntt/fntt_2d.cu, src/ntt/intt_2d.cu (negacyclic CT/GS,
 *                      output in bit-reversed order, fully reduced to [0,q))
 *   ModUp              src/rns_bconv.cu:530-628 and src/rns.cu:138-181 (digit limbs
 *                      copied unchanged, the rest base-converted without correction)
 *   inner product      src/eval_key_switch.cu:12-66 (key digit = [b | a] over QP)
 *   ModDown            src/rns_bconv.cu:776-828 (INTT of P limbs, fast base
 *                      conversion P->Ql, NTT, (cx - delta) * P^-1)
 *   key switch         src/eval_key_switch.cu:91-178
 *   Galois (NTT form)  include/galois.cuh:44-60 and src/galois.cu:8-21
 *   rescale            src/rns.cu:1125-1181 (floor: c_last mod q_j, no rounding term)
 *   tensor / add /     src/polymath.cu:17-230, 468-504; src/evaluate.cu:1237-1266
 *   multiply_plain
 *   ct-pt matmul       src/include/source/matrix_mul/Ct_pt_matrix_mul.cuh:112-158
 *                      (multiply_plain by a constant plaintext + add_inplace, summed)
 *
 * Layouts: a polynomial is [L][N] uint64 limbs (limb i under prime i of the
 * chain), a ciphertext is [2][L][N], a key-switching key is
 * [dnum][2][nq+np][N] with the "b" half first (the half added to c0).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

static inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }
static inline uint64_t addmod(uint64_t a, uint64_t b, uint64_t q) { uint64_t s = a + b; return s >= q ? s - q : s; }
static inline uint64_t submod(uint64_t a, uint64_t b, uint64_t q) { return a >= b ? a - b : a + q - b; }

static uint64_t powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = mulmod(r, a, q);
        a = mulmod(a, a, q);
        e >>= 1;
    }
    return r;
}

uint64_t orc_invmod(uint64_t a, uint64_t q) { return powmod(a % q, q - 2, q); }

/* Deterministic Miller-Rabin for 64-bit integers (these bases are exact below 2^64). */
int orc_is_prime(uint64_t n) {
    static const uint64_t bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    for (int i = 0; i < 12; i++) {
        if (n == bases[i]) return 1;
        if (n % bases[i] == 0) return 0;
    }
    uint64_t d = n - 1;
    int r = 0;
    while ((d & 1) == 0) { d >>= 1; r++; }
    for (int i = 0; i < 12; i++) {
        uint64_t x = powmod(bases[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int ok = 0;
        for (int k = 1; k < r; k++) {
            x = mulmod(x, x, n);
            if (x == n - 1) { ok = 1; break; }
        }
        if (!ok) return 0;
    }
    return 1;
}

/* CoeffModulus::Create restated: for each bit size, primes = 1 mod 2N searched
 * downwards from 2^b - 2N + 1; the i-th request of a size takes the LAST
 * remaining prime of that size's list.  Returns 0 on success. */
int orc_gen_primes(uint32_t log_n, const int *bits, uint32_t count, uint64_t *out) {
    uint64_t two_n = 2ull << log_n;
    for (uint32_t i = 0; i < count; i++) {
        int b = bits[i];
        uint32_t total = 0, before = 0;
        for (uint32_t k = 0; k < count; k++) {
            if (bits[k] == b) {
                total++;
                if (k < i) before++;
            }
        }
        /* the (before)-th request takes list[total - 1 - before] */
        uint32_t want = total - 1 - before;
        uint64_t v = (1ull << b) - two_n + 1, lower = 1ull << (b - 1);
        uint32_t found = 0;
        int got = 0;
        while (v > lower) {
            if (orc_is_prime(v)) {
                if (found == want) { out[i] = v; got = 1; break; }
                found++;
            }
            v -= two_n;
        }
        if (!got) return -1;
    }
    return 0;
}

static uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; i++) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

/* Smallest primitive 2N-th root of unity mod q (src/util/numth.cu:307-333 picks
 * a primitive root and scans all of its odd powers for the minimum). */
uint64_t orc_minimal_root(uint64_t q, uint32_t log_n) {
    uint64_t two_n = 2ull << log_n, n = 1ull << log_n;
    uint64_t root = 0;
    for (uint64_t x = 2; x < q; x++) {
        uint64_t r = powmod(x, (q - 1) / two_n, q);
        if (powmod(r, n, q) == q - 1) { root = r; break; }
    }
    uint64_t sq = mulmod(root, root, q), cur = root, best = root;
    for (uint64_t i = 0; i < n; i++) {
        if (cur < best) best = cur;
        cur = mulmod(cur, sq, q);
    }
    return best;
}

/* rp[bitrev(i)] = psi^i and irp[bitrev(i)] = psi^-i (no N^-1 folded in). */
void orc_ntt_tables(uint64_t q, uint32_t log_n, uint64_t *rp, uint64_t *irp) {
    uint32_t n = 1u << log_n;
    uint64_t psi = orc_minimal_root(q, log_n), ipsi = orc_invmod(psi, q);
    uint64_t p = 1, ip = 1;
    for (uint32_t i = 0; i < n; i++) {
        rp[bitrev(i, log_n)] = p;
        irp[bitrev(i, log_n)] = ip;
        p = mulmod(p, psi, q);
        ip = mulmod(ip, ipsi, q);
    }
}

/* Negacyclic forward NTT, natural order in, bit-reversed order out. */
void orc_ntt_fwd(uint64_t *a, uint32_t log_n, uint64_t q, const uint64_t *rp) {
    uint32_t n = 1u << log_n, t = n;
    for (uint32_t m = 1; m < n; m <<= 1) {
        t >>= 1;
        for (uint32_t i = 0; i < m; i++) {
            uint64_t w = rp[m + i];
            uint32_t j1 = 2 * i * t;
            for (uint32_t j = j1; j < j1 + t; j++) {
                uint64_t x = a[j], y = mulmod(a[j + t], w, q);
                a[j] = addmod(x, y, q);
                a[j + t] = submod(x, y, q);
            }
        }
    }
}

/* Inverse of orc_ntt_fwd (Gentleman-Sande), including the N^-1 scaling. */
void orc_ntt_inv(uint64_t *a, uint32_t log_n, uint64_t q, const uint64_t *irp) {
    uint32_t n = 1u << log_n, t = 1;
    for (uint32_t m = n >> 1; m >= 1; m >>= 1) {
        for (uint32_t i = 0; i < m; i++) {
            uint64_t w = irp[m + i];
            uint32_t j1 = 2 * i * t;
            for (uint32_t j = j1; j < j1 + t; j++) {
                uint64_t x = a[j], y = a[j + t];
                a[j] = addmod(x, y, q);
                a[j + t] = mulmod(submod(x, y, q), w, q);
            }
        }
        t <<= 1;
    }
    uint64_t ninv = orc_invmod(n, q);
    for (uint32_t j = 0; j < n; j++) a[j] = mulmod(a[j], ninv, q);
}

/* ------------------------------------------------------------------------- */
/* Context: prime chain Q (nq primes) followed by special primes P (np).     */

typedef struct {
    uint32_t log_n, n, nq, np;
    uint64_t *primes;   /* nq + np */
    uint64_t *rp, *irp; /* (nq + np) * n */
} orc_ctx;

orc_ctx *orc_ctx_create(uint32_t log_n, const uint64_t *primes, uint32_t nq, uint32_t np) {
    orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
    c->log_n = log_n;
    c->n = 1u << log_n;
    c->nq = nq;
    c->np = np;
    uint32_t k = nq + np;
    c->primes = (uint64_t *)malloc(sizeof(uint64_t) * k);
    memcpy(c->primes, primes, sizeof(uint64_t) * k);
    c->rp = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)k * c->n);
    c->irp = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)k * c->n);
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < (int)k; i++)
        orc_ntt_tables(primes[i], log_n, c->rp + (size_t)i * c->n, c->irp + (size_t)i * c->n);
    return c;
}

void orc_ctx_destroy(orc_ctx *c) {
    if (!c) return;
    free(c->primes);
    free(c->rp);
    free(c->irp);
    free(c);
}

void orc_ctx_tables(const orc_ctx *c, uint32_t prime_idx, uint64_t *rp, uint64_t *irp) {
    memcpy(rp, c->rp + (size_t)prime_idx * c->n, sizeof(uint64_t) * c->n);
    memcpy(irp, c->irp + (size_t)prime_idx * c->n, sizeof(uint64_t) * c->n);
}

/* Transform n_polys polynomials of L limbs each (Q chain, limb i -> prime i). */
void orc_ntt(const orc_ctx *c, uint64_t *a, uint32_t n_polys, uint32_t L, int inverse) {
    size_t n = c->n;
#pragma omp parallel for collapse(2) schedule(static)
    for (int p = 0; p < (int)n_polys; p++)
        for (int i = 0; i < (int)L; i++) {
            uint64_t *x = a + ((size_t)p * L + i) * n;
            if (inverse) orc_ntt_inv(x, c->log_n, c->primes[i], c->irp + (size_t)i * n);
            else orc_ntt_fwd(x, c->log_n, c->primes[i], c->rp + (size_t)i * n);
        }
}

/* Prime index (into c->primes) of extended limb j of a QlP polynomial. */
static inline uint32_t ext_prime(const orc_ctx *c, uint32_t L, uint32_t j) { return j < L ? j : c->nq + (j - L); }

void orc_add(const orc_ctx *c, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys, uint32_t L) {
    size_t n = c->n;
#pragma omp parallel for collapse(2)
    for (int p = 0; p < (int)n_polys; p++)
        for (int i = 0; i < (int)L; i++) {
            size_t o = ((size_t)p * L + i) * n;
            uint64_t q = c->primes[i];
            for (size_t k = 0; k < n; k++) out[o + k] = addmod(a[o + k], b[o + k], q);
        }
}

/* ct (n_polys x [L][N]) times one plaintext [L][N], pointwise (NTT form). */
void orc_multiply_plain(const orc_ctx *c, const uint64_t *ct, const uint64_t *pt, uint64_t *out, uint32_t n_polys,
                        uint32_t L) {
    size_t n = c->n;
#pragma omp parallel for collapse(2)
    for (int p = 0; p < (int)n_polys; p++)
        for (int i = 0; i < (int)L; i++) {
            size_t o = ((size_t)p * L + i) * n;
            uint64_t q = c->primes[i];
            for (size_t k = 0; k < n; k++) out[o + k] = mulmod(ct[o + k], pt[(size_t)i * n + k], q);
        }
}

/* (a0,a1) x (b0,b1) -> (a0b0, a0b1 + a1b0, a1b1) */
void orc_tensor(const orc_ctx *c, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t L) {
    size_t n = c->n, ln = (size_t)L * n;
#pragma omp parallel for
    for (int i = 0; i < (int)L; i++) {
        uint64_t q = c->primes[i];
        for (size_t k = 0; k < n; k++) {
            size_t o = (size_t)i * n + k;
            uint64_t a0 = a[o], a1 = a[ln + o], b0 = b[o], b1 = b[ln + o];
            out[o] = mulmod(a0, b0, q);
            out[ln + o] = addmod(mulmod(a0, b1, q), mulmod(a1, b0, q), q);
            out[2 * ln + o] = mulmod(a1, b1, q);
        }
    }
}

/* Floor rescale by the last prime: out_j = (c_j - NTT_j(c_last mod q_j)) * q_last^-1. */
void orc_rescale(const orc_ctx *c, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L) {
    size_t n = c->n;
    uint64_t ql = c->primes[L - 1];
    uint64_t *last = (uint64_t *)malloc(sizeof(uint64_t) * n * n_polys);
    for (uint32_t p = 0; p < n_polys; p++) {
        memcpy(last + p * n, in + ((size_t)p * L + L - 1) * n, sizeof(uint64_t) * n);
        orc_ntt_inv(last + p * n, c->log_n, ql, c->irp + (size_t)(L - 1) * n);
    }
#pragma omp parallel for collapse(2)
    for (int p = 0; p < (int)n_polys; p++)
        for (int j = 0; j < (int)L - 1; j++) {
            uint64_t qj = c->primes[j], inv = orc_invmod(ql % qj, qj);
            uint64_t *o = out + ((size_t)p * (L - 1) + j) * n;
            for (size_t k = 0; k < n; k++) o[k] = last[p * n + k] % qj;
            orc_ntt_fwd(o, c->log_n, qj, c->rp + (size_t)j * n);
            const uint64_t *ci = in + ((size_t)p * L + j) * n;
            for (size_t k = 0; k < n; k++) o[k] = mulmod(submod(ci[k], o[k], qj), inv, qj);
        }
    free(last);
}

/* NTT-domain automorphism X -> X^elt: out[k] = in[perm[k]] with
 * 2*brv(perm[k]) + 1 = (2*brv(k) + 1) * elt mod 2N. */
void orc_galois_perm(uint32_t log_n, uint32_t elt, uint32_t *perm) {
    uint32_t n = 1u << log_n;
    for (uint32_t k = 0; k < n; k++) {
        uint64_t e = ((uint64_t)(2 * bitrev(k, log_n) + 1) * elt) & (2ull * n - 1);
        perm[k] = bitrev((uint32_t)((e - 1) >> 1), log_n);
    }
}

void orc_apply_galois(const orc_ctx *c, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
                      uint32_t elt) {
    size_t n = c->n;
    uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * n);
    orc_galois_perm(c->log_n, elt, perm);
#pragma omp parallel for
    for (int r = 0; r < (int)(n_polys * L); r++)
        for (size_t k = 0; k < n; k++) out[(size_t)r * n + k] = in[(size_t)r * n + perm[k]];
    free(perm);
}

/* Galois element of a left rotation by `step` slots (src/galois.cu:47-91). */
uint32_t orc_galois_elt_from_step(uint32_t log_n, int step) {
    uint32_t n = 1u << log_n;
    uint64_t m = 2ull * n;
    if (step == 0) return (uint32_t)(m - 1);
    uint32_t pos = (uint32_t)(step < 0 ? -step : step);
    int s = step < 0 ? (int)(n >> 1) - (int)pos : (int)pos;
    uint64_t g = 1;
    while (s--) g = (g * 5) & (m - 1);
    return (uint32_t)g;
}

/* ModUp of c (NTT form, L limbs): out[b] is digit b extended to QlP
 * ([beta][L+np][N]).  Digit b covers limbs [b*np, min((b+1)*np, L)). */
void orc_modup(const orc_ctx *c, const uint64_t *cin, uint32_t L, uint64_t *out) {
    size_t n = c->n;
    uint32_t alpha = c->np, beta = (L + alpha - 1) / alpha, LP = L + c->np;
    uint64_t *x = (uint64_t *)malloc(sizeof(uint64_t) * L * n);
    memcpy(x, cin, sizeof(uint64_t) * L * n);
#pragma omp parallel for
    for (int i = 0; i < (int)L; i++) orc_ntt_inv(x + (size_t)i * n, c->log_n, c->primes[i], c->irp + (size_t)i * n);
    for (uint32_t b = 0; b < beta; b++) {
        uint32_t s = b * alpha, e = s + alpha < L ? s + alpha : L;
        /* y_i = x_i * (Qhat_i)^-1 mod q_i, Qhat_i = prod_{k in digit, k != i} q_k */
        for (uint32_t i = s; i < e; i++) {
            uint64_t qi = c->primes[i], h = 1;
            for (uint32_t k = s; k < e; k++)
                if (k != i) h = mulmod(h, c->primes[k] % qi, qi);
            uint64_t hinv = orc_invmod(h, qi);
            for (size_t k = 0; k < n; k++) x[(size_t)i * n + k] = mulmod(x[(size_t)i * n + k], hinv, qi);
        }
        uint64_t *ob = out + (size_t)b * LP * n;
#pragma omp parallel for
        for (int j = 0; j < (int)LP; j++) {
            uint64_t *o = ob + (size_t)j * n;
            if (j >= (int)s && j < (int)e) {
                memcpy(o, cin + (size_t)j * n, sizeof(uint64_t) * n);
                continue;
            }
            uint32_t pj = ext_prime(c, L, j);
            uint64_t t = c->primes[pj];
            uint64_t hm[64];
            for (uint32_t i = s; i < e; i++) {
                uint64_t h = 1;
                for (uint32_t k = s; k < e; k++)
                    if (k != i) h = mulmod(h, c->primes[k] % t, t);
                hm[i - s] = h;
            }
            for (size_t k = 0; k < n; k++) {
                u128 acc = 0;
                for (uint32_t i = s; i < e; i++) acc += (u128)x[(size_t)i * n + k] * hm[i - s];
                o[k] = (uint64_t)(acc % t);
            }
            orc_ntt_fwd(o, c->log_n, t, c->rp + (size_t)pj * n);
        }
    }
    free(x);
}

/* ModDown of one QlP polynomial (NTT form) to Ql: (cx_j - NTT(conv_P->q_j(INTT(cx_P)))) * P^-1. */
static void moddown_one(const orc_ctx *c, const uint64_t *cx, uint32_t L, uint64_t *out) {
    size_t n = c->n;
    uint32_t np = c->np;
    uint64_t *z = (uint64_t *)malloc(sizeof(uint64_t) * np * n);
    for (uint32_t k = 0; k < np; k++) {
        uint32_t pk = c->nq + k;
        uint64_t p = c->primes[pk], h = 1;
        memcpy(z + (size_t)k * n, cx + (size_t)(L + k) * n, sizeof(uint64_t) * n);
        orc_ntt_inv(z + (size_t)k * n, c->log_n, p, c->irp + (size_t)pk * n);
        for (uint32_t k2 = 0; k2 < np; k2++)
            if (k2 != k) h = mulmod(h, c->primes[c->nq + k2] % p, p);
        uint64_t hinv = orc_invmod(h, p);
        for (size_t t = 0; t < n; t++) z[(size_t)k * n + t] = mulmod(z[(size_t)k * n + t], hinv, p);
    }
#pragma omp parallel for
    for (int j = 0; j < (int)L; j++) {
        uint64_t q = c->primes[j];
        uint64_t hm[64], P = 1;
        for (uint32_t k = 0; k < np; k++) {
            uint64_t h = 1;
            for (uint32_t k2 = 0; k2 < np; k2++)
                if (k2 != k) h = mulmod(h, c->primes[c->nq + k2] % q, q);
            hm[k] = h;
            P = mulmod(P, c->primes[c->nq + k] % q, q);
        }
        uint64_t pinv = orc_invmod(P, q);
        uint64_t *o = out + (size_t)j * n;
        for (size_t t = 0; t < n; t++) {
            u128 acc = 0;
            for (uint32_t k = 0; k < np; k++) acc += (u128)z[(size_t)k * n + t] * hm[k];
            o[t] = (uint64_t)(acc % q);
        }
        orc_ntt_fwd(o, c->log_n, q, c->rp + (size_t)j * n);
        const uint64_t *ci = cx + (size_t)j * n;
        for (size_t t = 0; t < n; t++) o[t] = mulmod(submod(ci[t], o[t], q), pinv, q);
    }
    free(z);
}

/* The key switch's inner product: cx [2][L + np][N] = sum_b ModUp(d)_b * key_b over QlP,
 * before the ModDown (keyswitch_inplace up to the inner product, eval_key_switch.cu:91-160). */
static void keyswitch_acc(const orc_ctx *c, const uint64_t *d, uint32_t L, const uint64_t *key, uint64_t *cx) {
    size_t n = c->n;
    uint32_t alpha = c->np, beta = (L + alpha - 1) / alpha, LP = L + c->np, QP = c->nq + c->np;
    uint64_t *up = (uint64_t *)malloc(sizeof(uint64_t) * beta * LP * n);
    orc_modup(c, d, L, up);
#pragma omp parallel for
    for (int j = 0; j < (int)LP; j++) {
        uint32_t pj = ext_prime(c, L, j);
        uint64_t t = c->primes[pj];
        for (size_t k = 0; k < n; k++) {
            u128 a0 = 0, a1 = 0;
            for (uint32_t b = 0; b < beta; b++) {
                uint64_t v = up[((size_t)b * LP + j) * n + k];
                const uint64_t *kb = key + (size_t)b * 2 * QP * n;
                a0 += (u128)v * kb[(size_t)pj * n + k];
                a1 += (u128)v * kb[((size_t)QP + pj) * n + k];
                a0 %= t;
                a1 %= t;
            }
            cx[(size_t)j * n + k] = (uint64_t)a0;
            cx[((size_t)LP + j) * n + k] = (uint64_t)a1;
        }
    }
    free(up);
}

/* Hybrid key switch of one polynomial d (NTT form, L limbs) with a key of
 * dnum digits over QP: returns (cx0, cx1), each [L][N], not yet added. */
void orc_keyswitch(const orc_ctx *c, const uint64_t *d, uint32_t L, const uint64_t *key, uint32_t dnum,
                   uint64_t *out) {
    size_t n = c->n;
    uint32_t LP = L + c->np;
    (void)dnum;
    uint64_t *cx = (uint64_t *)malloc(sizeof(uint64_t) * 2 * LP * n);
    keyswitch_acc(c, d, L, key, cx);
    moddown_one(c, cx, L, out);
    moddown_one(c, cx + (size_t)LP * n, L, out + (size_t)L * n);
    free(cx);
}

/* ModDown of one extended polynomial y [L + np][N] (NTT form over QlP) by S = q_{L-1} P
 * into out [L-1][N] = floor(y / S): z_k = INTT(y_{s_k}) (S/s_k)^-1 mod s_k for
 * s = (q_{L-1}, p_0, ..), v = floor(sum_k z_k / s_k) in double precision (one unfused
 * multiply and add per term, k in order), conv_j = (sum_k z_k (S/s_k) - v S) mod q_j = [y]_S
 * mod q_j, out_j = (y_j - NTT(conv_j)) S^-1 mod q_j.  The conversion of moddown_from_NTT
 * (rns_bconv.cu:776-828) with q_{L-1} counted among the special primes, made exact by
 * the overflow count v. */
static void moddown_s(const orc_ctx *c, const uint64_t *y, uint32_t L, uint64_t *out) {
    size_t n = c->n;
    uint32_t ns = c->np + 1;
    uint32_t sidx[65];
    sidx[0] = L - 1;
    for (uint32_t k = 0; k < c->np; k++) sidx[1 + k] = c->nq + k;
    uint64_t *z = (uint64_t *)malloc(sizeof(uint64_t) * ns * n);
    for (uint32_t k = 0; k < ns; k++) {
        uint64_t s = c->primes[sidx[k]], h = 1;
        uint32_t row = k == 0 ? L - 1 : L + (k - 1);
        memcpy(z + (size_t)k * n, y + (size_t)row * n, sizeof(uint64_t) * n);
        orc_ntt_inv(z + (size_t)k * n, c->log_n, s, c->irp + (size_t)sidx[k] * n);
        for (uint32_t k2 = 0; k2 < ns; k2++)
            if (k2 != k) h = mulmod(h, c->primes[sidx[k2]] % s, s);
        uint64_t hinv = orc_invmod(h, s);
        for (size_t t = 0; t < n; t++) z[(size_t)k * n + t] = mulmod(z[(size_t)k * n + t], hinv, s);
    }
    uint8_t *v = (uint8_t *)malloc(n);
    double inv_s[65];
    for (uint32_t k = 0; k < ns; k++) inv_s[k] = 1.0 / (double)c->primes[sidx[k]];
    for (size_t t = 0; t < n; t++) {
        double f = 0.0;
        for (uint32_t k = 0; k < ns; k++) {
            double prod = (double)z[(size_t)k * n + t] * inv_s[k];
            f = f + prod;
        }
        v[t] = (uint8_t)f;
    }
#pragma omp parallel for
    for (int j = 0; j < (int)L - 1; j++) {
        uint64_t q = c->primes[j];
        uint64_t hm[65], S = 1;
        for (uint32_t k = 0; k < ns; k++) {
            uint64_t h = 1;
            for (uint32_t k2 = 0; k2 < ns; k2++)
                if (k2 != k) h = mulmod(h, c->primes[sidx[k2]] % q, q);
            hm[k] = h;
            S = mulmod(S, c->primes[sidx[k]] % q, q);
        }
        uint64_t sinv = orc_invmod(S, q);
        uint64_t *o = out + (size_t)j * n;
        for (size_t t = 0; t < n; t++) {
            u128 acc = 0;
            for (uint32_t k = 0; k < ns; k++) acc += (u128)z[(size_t)k * n + t] * hm[k];
            o[t] = submod((uint64_t)(acc % q), mulmod(v[t], S, q), q);
        }
        orc_ntt_fwd(o, c->log_n, q, c->rp + (size_t)j * n);
        const uint64_t *yi = y + (size_t)j * n;
        for (size_t t = 0; t < n; t++) o[t] = mulmod(submod(yi[t], o[t], q), sinv, q);
    }
    free(v);
    free(z);
}

/* Relinearize and rescale one size-3 ciphertext ct3 [3][L][N] (L >= 2) into out [2][L-1][N]
 * in one ModDown: y_h = P c_h + cx_h over QlP, out_h = ModDown_S(y_h) with S = q_{L-1} P. */
void orc_relin_rescale(const orc_ctx *c, const uint64_t *ct3, uint32_t L, const uint64_t *key, uint64_t *out) {
    size_t n = c->n, ln = (size_t)L * n;
    uint32_t LP = L + c->np;
    uint64_t *cx = (uint64_t *)malloc(sizeof(uint64_t) * 2 * LP * n);
    keyswitch_acc(c, ct3 + 2 * ln, L, key, cx);
    for (uint32_t h = 0; h < 2; h++) {
        uint64_t *y = cx + (size_t)h * LP * n;
        for (uint32_t j = 0; j < L; j++) {
            uint64_t q = c->primes[j], P = 1;
            for (uint32_t k = 0; k < c->np; k++) P = mulmod(P, c->primes[c->nq + k] % q, q);
            const uint64_t *cj = ct3 + (size_t)h * ln + (size_t)j * n;
            for (size_t t = 0; t < n; t++) y[(size_t)j * n + t] = addmod(y[(size_t)j * n + t], mulmod(P, cj[t], q), q);
        }
        moddown_s(c, y, L, out + (size_t)h * (L - 1) * n);
    }
    free(cx);
}


/* Hoisted Galois key switching (Halevi-Shoup): ModUp of c1 once, then for each
 * element g the automorphism is applied to the extended digits (an NTT-domain
 * permutation of every limb), followed by the inner product with g's key and
 * ModDown: out_g = (sigma_g(c0) + cx0, cx1).  keys[e] -> [dnum][2][QP][N],
 * outs[e] -> [2][L][N]. */
void orc_apply_galois_hoisted(const orc_ctx *c, const uint64_t *ct, uint32_t L, uint32_t n_elts,
                              const uint32_t *elts, const uint64_t *const *keys, uint32_t dnum, uint64_t *const *outs) {
    size_t n = c->n, ln = (size_t)L * n;
    uint32_t alpha = c->np, beta = (L + alpha - 1) / alpha, LP = L + c->np, QP = c->nq + c->np;
    (void)dnum;
    uint64_t *up = (uint64_t *)malloc(sizeof(uint64_t) * beta * LP * n);
    orc_modup(c, ct + ln, L, up);
    uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint64_t *cx = (uint64_t *)malloc(sizeof(uint64_t) * 2 * LP * n);
    for (uint32_t e = 0; e < n_elts; e++) {
        orc_galois_perm(c->log_n, elts[e], perm);
        const uint64_t *key = keys[e];
#pragma omp parallel for
        for (int j = 0; j < (int)LP; j++) {
            uint32_t pj = ext_prime(c, L, j);
            uint64_t t = c->primes[pj];
            for (size_t k = 0; k < n; k++) {
                u128 a0 = 0, a1 = 0;
                for (uint32_t b = 0; b < beta; b++) {
                    uint64_t v = up[((size_t)b * LP + j) * n + perm[k]];
                    const uint64_t *kb = key + (size_t)b * 2 * QP * n;
                    a0 = (a0 + (u128)v * kb[(size_t)pj * n + k]) % t;
                    a1 = (a1 + (u128)v * kb[((size_t)QP + pj) * n + k]) % t;
                }
                cx[(size_t)j * n + k] = (uint64_t)a0;
                cx[((size_t)LP + j) * n + k] = (uint64_t)a1;
            }
        }
        uint64_t *out = outs[e];
        moddown_one(c, cx, L, out);
        moddown_one(c, cx + (size_t)LP * n, L, out + ln);
        /* out0 += sigma(c0) */
#pragma omp parallel for
        for (int i = 0; i < (int)L; i++) {
            uint64_t q = c->primes[i];
            for (size_t k = 0; k < n; k++)
                out[(size_t)i * n + k] = addmod(out[(size_t)i * n + k], ct[(size_t)i * n + perm[k]], q);
        }
    }
    free(cx);
    free(perm);
    free(up);
}

/* ---------------- shared-a batches (multi-secret RLWE) -----------------------
 * One group = [n+1][L][N] = (b_0 .. b_{n-1}, a), b_i + a s'_i ~ m_i
 * (src/include/source/bootstrapping/SharedACiphertext.cuh:9-21).                */

/* inner products of the extended digits ext [beta][LP][N] (read at perm[k]) with
 * key halves key [beta][H][QP][N] -> cx [H][LP][N] */
static void ip_multi(const orc_ctx *c, const uint64_t *ext, uint32_t beta, uint32_t L, const uint64_t *key, uint32_t H,
                     const uint32_t *perm, uint64_t *cx) {
    size_t n = c->n;
    uint32_t LP = L + c->np, QP = c->nq + c->np;
#pragma omp parallel for
    for (int j = 0; j < (int)LP; j++) {
        uint32_t pj = ext_prime(c, L, j);
        uint64_t t = c->primes[pj];
        for (size_t k = 0; k < n; k++) {
            size_t ks = perm ? perm[k] : k;
            for (uint32_t h = 0; h < H; h++) {
                u128 a = 0;
                for (uint32_t b = 0; b < beta; b++)
                    a = (a + (u128)ext[((size_t)b * LP + j) * n + ks] *
                                 key[(((size_t)b * H + h) * QP + pj) * n + k]) % t;
                cx[((size_t)h * LP + j) * n + k] = (uint64_t)a;
            }
        }
    }
}

/* Sh-Rot (ShRotate.cu:201-257), hoisted over several elements: one ModUp of a, then per
 * element g: b'_i = sigma_g(b_i) + ModDown(<up, B_i>), a' = ModDown(<up, A>).
 * keys[e]: [dnum][n+1][QP][N]; outs[e]: [n+1][L][N]. */
void orc_shared_rotate_hoisted(const orc_ctx *c, const uint64_t *sh, uint32_t n_mem, uint32_t L, uint32_t n_elts,
                               const uint32_t *elts, const uint64_t *const *keys, uint64_t *const *outs) {
    size_t n = c->n, ln = (size_t)L * n;
    uint32_t alpha = c->np, beta = (L + alpha - 1) / alpha, LP = L + c->np, H = n_mem + 1;
    uint64_t *up = (uint64_t *)malloc(sizeof(uint64_t) * beta * LP * n);
    orc_modup(c, sh + (size_t)n_mem * ln, L, up);
    uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint64_t *cx = (uint64_t *)malloc(sizeof(uint64_t) * H * LP * n);
    for (uint32_t e = 0; e < n_elts; e++) {
        orc_galois_perm(c->log_n, elts[e], perm);
        ip_multi(c, up, beta, L, keys[e], H, perm, cx);
        for (uint32_t h = 0; h < H; h++) {
            uint64_t *o = outs[e] + (size_t)h * ln;
            moddown_one(c, cx + (size_t)h * LP * n, L, o);
            if (h < n_mem) {
                const uint64_t *b = sh + (size_t)h * ln;
                for (uint32_t i = 0; i < L; i++)
                    for (size_t k = 0; k < n; k++)
                        o[(size_t)i * n + k] = addmod(o[(size_t)i * n + k], b[(size_t)i * n + perm[k]], c->primes[i]);
            }
        }
    }
    free(cx);
    free(perm);
    free(up);
}

/* ---------------- the extended basis QlP (double hoisting) ----------------
 * An extended polynomial at level L has L + np limbs (Q limbs, then the special primes) and
 * stands for its ModDown (Bossuat et al., double hoisting of BSGS key switches). */

static uint64_t p_mod_q(const orc_ctx *c, uint64_t q) {
    uint64_t P = 1;
    for (uint32_t k = 0; k < c->np; k++) P = mulmod(P, c->primes[c->nq + k] % q, q);
    return P;
}

/* out = P * in on the Q limbs, 0 on the special-prime limbs */
void orc_extend(const orc_ctx *c, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L) {
    size_t n = c->n;
    uint32_t LP = L + c->np;
    for (uint32_t p = 0; p < n_polys; p++)
        for (uint32_t j = 0; j < LP; j++) {
            uint64_t *o = out + ((size_t)p * LP + j) * n;
            if (j >= L) {
                memset(o, 0, sizeof(uint64_t) * n);
                continue;
            }
            uint64_t q = c->primes[j], P = p_mod_q(c, q);
            const uint64_t *x = in + ((size_t)p * L + j) * n;
            for (size_t k = 0; k < n; k++) o[k] = mulmod(x[k], P, q);
        }
}

void orc_moddown_ext(const orc_ctx *c, const uint64_t *ext, uint64_t *out, uint32_t n_polys, uint32_t L) {
    size_t n = c->n;
    uint32_t LP = L + c->np;
    for (uint32_t p = 0; p < n_polys; p++) moddown_one(c, ext + (size_t)p * LP * n, L, out + (size_t)p * L * n);
}

/* Sh-Rot with extended outputs: the input group is [n+1][L][N] (in_ext = 0) or extended
 * [n+1][L+np][N] (in_ext = 1: its a row is brought down first); per element e,
 * outs[e][h] = <up, key_h> over QlP, plus for the b rows sigma(b) scaled by P (ordinary input)
 * or sigma(b_ext) (extended input). */
void orc_shared_rotate_ext(const orc_ctx *c, const uint64_t *in, int in_ext, uint32_t n_mem, uint32_t L,
                           uint32_t n_elts, const uint32_t *elts, const uint64_t *const *keys, uint64_t *const *outs) {
    size_t n = c->n;
    uint32_t alpha = c->np, beta = (L + alpha - 1) / alpha, LP = L + c->np, H = n_mem + 1;
    size_t rowl = (size_t)(in_ext ? LP : L) * n;
    uint64_t *up = (uint64_t *)malloc(sizeof(uint64_t) * beta * LP * n);
    if (in_ext) {
        uint64_t *aq = (uint64_t *)malloc(sizeof(uint64_t) * L * n);
        moddown_one(c, in + (size_t)n_mem * rowl, L, aq);
        orc_modup(c, aq, L, up);
        free(aq);
    } else {
        orc_modup(c, in + (size_t)n_mem * rowl, L, up);
    }
    uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * n);
    for (uint32_t e = 0; e < n_elts; e++) {
        orc_galois_perm(c->log_n, elts[e], perm);
        ip_multi(c, up, beta, L, keys[e], H, perm, outs[e]);
        for (uint32_t h = 0; h < n_mem; h++)
            for (uint32_t j = 0; j < LP; j++) {
                if (!in_ext && j >= L) continue;
                uint64_t q = c->primes[ext_prime(c, L, j)], P = in_ext ? 1 : p_mod_q(c, q);
                const uint64_t *b = in + (size_t)h * rowl + (size_t)j * n;
                uint64_t *o = outs[e] + ((size_t)h * LP + j) * n;
                for (size_t k = 0; k < n; k++) o[k] = addmod(o[k], mulmod(b[perm[k]], P, q), q);
            }
    }
    free(perm);
    free(up);
}

/* Exact extension of a (NTT form, L limbs) to QlP: the Ql rows keep a, the P rows get
 * (sum_i y_i qhat_i - v Q) mod p_k with y_i = [x_i qhat_i^-1]_{q_i} (x = INTT(a)) and
 * v = floor(sum_i y_i / q_i) in double arithmetic as FmtSwitch.cu:86-106 computes it: the
 * quotients y_i / q_i summed in limb order, truncated, and raised by one where the sum is
 * within 1e-9 below the next integer. */
static void exact_extend(const orc_ctx *c, const uint64_t *a, uint32_t L, uint64_t *ext) {
    size_t n = c->n;
    uint32_t LP = L + c->np;
    uint64_t *y = (uint64_t *)malloc(sizeof(uint64_t) * L * n);
    memcpy(y, a, sizeof(uint64_t) * L * n);
    memcpy(ext, a, sizeof(uint64_t) * L * n);
    for (uint32_t i = 0; i < L; i++) {
        uint64_t qi = c->primes[i], h = 1;
        orc_ntt_inv(y + (size_t)i * n, c->log_n, qi, c->irp + (size_t)i * n);
        for (uint32_t k = 0; k < L; k++)
            if (k != i) h = mulmod(h, c->primes[k] % qi, qi);
        uint64_t hinv = orc_invmod(h, qi);
        for (size_t t = 0; t < n; t++) y[(size_t)i * n + t] = mulmod(y[(size_t)i * n + t], hinv, qi);
    }
#pragma omp parallel for
    for (int kk = 0; kk < (int)c->np; kk++) {
        uint32_t pk = c->nq + kk;
        uint64_t p = c->primes[pk], Qm = 1, hm[64];
        for (uint32_t i = 0; i < L; i++) {
            uint64_t h = 1;
            for (uint32_t k = 0; k < L; k++)
                if (k != i) h = mulmod(h, c->primes[k] % p, p);
            hm[i] = h;
            Qm = mulmod(Qm, c->primes[i] % p, p);
        }
        uint64_t *o = ext + (size_t)(L + kk) * n;
        for (size_t t = 0; t < n; t++) {
            double frac = 0.0;
            u128 acc = 0;
            for (uint32_t i = 0; i < L; i++) {
                uint64_t yi = y[(size_t)i * n + t];
                frac = frac + (double)yi / (double)c->primes[i];
                acc += (u128)yi * hm[i];
            }
            uint64_t v = (uint64_t)frac;
            if (frac - (double)v > 1.0 - 1e-9) v += 1;
            o[t] = submod((uint64_t)(acc % p), mulmod(v, Qm, p), p);
        }
        orc_ntt_fwd(o, c->log_n, p, c->rp + (size_t)pk * n);
    }
    (void)LP;
    free(y);
}

/* ModRaise (Bootstrapper.cu:3271-3356, SharedABatchOps.cu:15-25, 128-166): one-limb polynomials
 * [n_polys][N] (mod q0, NTT form) -> [n_polys][L][N] (NTT form) by the centred lift: the residue x
 * mod q0 goes to every prime as x, or as x - q0 when x > floor(q0 / 2). */
void orc_modraise(const orc_ctx *c, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L) {
    size_t n = c->n;
    uint64_t q0 = c->primes[0], *x = (uint64_t *)malloc(n * 8);
    for (uint32_t p = 0; p < n_polys; p++) {
        memcpy(x, in + (size_t)p * n, n * 8);
        orc_ntt_inv(x, c->log_n, q0, c->irp);
        for (uint32_t j = 0; j < L; j++) {
            uint64_t qj = c->primes[j], *o = out + ((size_t)p * L + j) * n;
            for (size_t k = 0; k < n; k++) o[k] = x[k] > q0 / 2 ? submod(x[k] % qj, q0 % qj, qj) : x[k] % qj;
        }
    }
    free(x);
    orc_ntt(c, out, n_polys, L, 0);
}

/* The exact extension alone, for n_polys polynomials [n_polys][L][N] (NTT form) into
 * [n_polys][L + np][N] (the extension step of FmtSwitch.cu:317-329). */
void orc_exact_extend(const orc_ctx *c, const uint64_t *a, uint32_t n_polys, uint32_t L, uint64_t *ext) {
    size_t n = c->n;
    for (uint32_t p = 0; p < n_polys; p++)
        exact_extend(c, a + (size_t)p * L * n, L, ext + (size_t)p * (L + c->np) * n);
}

/* FmtSwitch forward (FmtSwitch.cu:276-394) of one group: cts [n][2][L][N] under s ->
 * out [n+1][L][N] under s'_i with key [n][n+1][QP][N] (B_fmt[j][i], a_fmt[j]). */
void orc_fmt_forward(const orc_ctx *c, const uint64_t *cts, uint32_t n_mem, uint32_t L, const uint64_t *key,
                     uint64_t *out) {
    size_t n = c->n, ln = (size_t)L * n;
    uint32_t LP = L + c->np, H = n_mem + 1;
    uint64_t *ext = (uint64_t *)malloc(sizeof(uint64_t) * n_mem * LP * n);
    for (uint32_t j = 0; j < n_mem; j++) exact_extend(c, cts + ((size_t)j * 2 + 1) * ln, L, ext + (size_t)j * LP * n);
    uint64_t *cx = (uint64_t *)malloc(sizeof(uint64_t) * H * LP * n);
    ip_multi(c, ext, n_mem, L, key, H, NULL, cx);
    for (uint32_t h = 0; h < H; h++) {
        uint64_t *o = out + (size_t)h * ln;
        moddown_one(c, cx + (size_t)h * LP * n, L, o);
        if (h < n_mem) orc_add(c, o, cts + (size_t)h * 2 * ln, o, 1, L);
    }
    free(cx);
    free(ext);
}

/* FmtSwitch backward (FmtSwitch.cu:396-429) of one group, hoisted: one ModUp of a, then
 * member i -> (b_i + cx0, cx1) with keys[i] [dnum][2][QP][N]; out [n][2][L][N]. */
void orc_fmt_backward(const orc_ctx *c, const uint64_t *sh, uint32_t n_mem, uint32_t L, const uint64_t *const *keys,
                      uint64_t *out) {
    size_t n = c->n, ln = (size_t)L * n;
    uint32_t alpha = c->np, beta = (L + alpha - 1) / alpha, LP = L + c->np;
    uint64_t *up = (uint64_t *)malloc(sizeof(uint64_t) * beta * LP * n);
    orc_modup(c, sh + (size_t)n_mem * ln, L, up);
    uint64_t *cx = (uint64_t *)malloc(sizeof(uint64_t) * 2 * LP * n);
    for (uint32_t i = 0; i < n_mem; i++) {
        ip_multi(c, up, beta, L, keys[i], 2, NULL, cx);
        uint64_t *o = out + (size_t)i * 2 * ln;
        moddown_one(c, cx, L, o);
        moddown_one(c, cx + (size_t)LP * n, L, o + ln);
        orc_add(c, o, sh + (size_t)i * ln, o, 1, L);
    }
    free(cx);
    free(up);
}

/* Relinearize a size-3 ciphertext: (c0 + cx0, c1 + cx1) with cx = KS(c2). */
void orc_relinearize(const orc_ctx *c, const uint64_t *ct3, uint32_t L, const uint64_t *key, uint32_t dnum,
                     uint64_t *out) {
    size_t ln = (size_t)L * c->n;
    uint64_t *cx = (uint64_t *)malloc(sizeof(uint64_t) * 2 * ln);
    orc_keyswitch(c, ct3 + 2 * ln, L, key, dnum, cx);
    orc_add(c, ct3, cx, out, 2, L);
    free(cx);
}

/* Rotation / conjugation: (sigma(c0) + cx0, cx1) with cx = KS(sigma(c1)). */
void orc_apply_galois_ct(const orc_ctx *c, const uint64_t *ct, uint32_t L, uint32_t elt, const uint64_t *key,
                         uint32_t dnum, uint64_t *out) {
    size_t ln = (size_t)L * c->n;
    uint64_t *g = (uint64_t *)malloc(sizeof(uint64_t) * 2 * ln);
    uint64_t *cx = (uint64_t *)malloc(sizeof(uint64_t) * 2 * ln);
    orc_apply_galois(c, ct, g, 2, L, elt);
    orc_keyswitch(c, g + ln, L, key, dnum, cx);
    orc_add(c, g, cx, out, 1, L);
    memcpy(out + ln, cx + ln, sizeof(uint64_t) * ln);
    free(cx);
    free(g);
}

/* Signed integer -> residue (the canonical form an NTT-domain constant takes). */
static inline uint64_t signed_residue(int64_t w, uint64_t q) {
    if (w >= 0) return (uint64_t)w % q;
    uint64_t r = (uint64_t)(-(w + 1)) % q; /* |w| - 1 without overflow */
    r = r + 1 == q ? 0 : r + 1;
    return r ? q - r : 0;
}

uint64_t orc_signed_residue(int64_t w, uint64_t q) { return signed_residue(w, q); }

/* Y_o = sum_i X_i * W[i][o] (constant plaintexts, NTT form), no rescale.
 * X: [n_in][2][L][N]; W: [n_in][n_out] signed integers; Y: [n_out][2][L][N]. */
void orc_ctpt_matmul(const orc_ctx *c, const uint64_t *X, const int64_t *W, uint32_t n_in, uint32_t n_out,
                     uint32_t L, uint64_t *Y) {
    size_t n = c->n, ctw = 2 * (size_t)L * n;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int o = 0; o < (int)n_out; o++)
        for (int r = 0; r < (int)(2 * L); r++) {
            uint32_t limb = (uint32_t)r % L;
            uint64_t q = c->primes[limb];
            uint64_t *y = Y + (size_t)o * ctw + (size_t)r * n;
            u128 *acc = (u128 *)calloc(n, sizeof(u128));
            for (uint32_t i = 0; i < n_in; i++) {
                uint64_t w = signed_residue(W[(size_t)i * n_out + o], q);
                const uint64_t *x = X + (size_t)i * ctw + (size_t)r * n;
                for (size_t k = 0; k < n; k++) {
                    acc[k] += (u128)x[k] * w;
                    if ((i & 31) == 31) acc[k] %= q;
                }
            }
            for (size_t k = 0; k < n; k++) y[k] = (uint64_t)(acc[k] % q);
            free(acc);
        }
}
