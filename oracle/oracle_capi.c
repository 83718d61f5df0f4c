/* TEST INFRASTRUCTURE ONLY.  The CPU oracle behind the C ABI of include/shmoai_ckks.h:
 * every entry point the C++ host library (include/shmoai/host.hpp) calls, implemented on
 * host memory with the oracle's restatement of the reference arithmetic (ckks_oracle.c).
 * oracle/Makefile links the host library's unchanged sources against this file to get
 * the whole pipeline (key generation, evaluator, bootstrapping) on the CPU, which the
 * tests compare bit for bit with the same pipeline on the CUDA library.  Nothing in the
 * product links or loads it.
 *
 * "Device" memory is host memory here; streams and workspaces are ignored.  The samplers
 * use the same counter-based function as the CUDA library (splitmix64's output mix of
 * seed + (index + 1) * golden gamma), so keys and ciphertexts are identical. */
#include <math.h>
#include <stdio.h>

#include "ckks_oracle.c"

#include "../include/shmoai_ckks.h"

struct shm_context {
    orc_ctx *c;
    uint32_t dnum;
};

static __thread char g_err[256];

static int fail(const char *msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return SHM_EINVAL;
}

const char *shm_last_error(void) { return g_err; }
uint64_t shm_kernel_launches(void) { return 0; }

static int make_ctx(shm_context **out, uint32_t log_n, const uint64_t *primes, uint32_t nq, uint32_t np) {
    if (!out) return fail("null output");
    if (log_n != 12 && log_n != 16) return fail("log_n must be 12 or 16");
    shm_context *h = (shm_context *)calloc(1, sizeof(shm_context));
    h->c = orc_ctx_create(log_n, primes, nq, np);
    h->dnum = np ? nq / np : 0;
    *out = h;
    return SHM_OK;
}

int shm_context_create(shm_context **out, uint32_t log_n, const int *bits, uint32_t n_q, uint32_t n_p, int device) {
    (void)device;
    uint64_t *p = (uint64_t *)malloc(sizeof(uint64_t) * (n_q + n_p));
    if (orc_gen_primes(log_n, bits, n_q + n_p, p) != 0) {
        free(p);
        return fail("not enough primes");
    }
    int rc = make_ctx(out, log_n, p, n_q, n_p);
    free(p);
    return rc;
}

int shm_context_create_from_primes(shm_context **out, uint32_t log_n, const uint64_t *primes, uint32_t n_q,
                                   uint32_t n_p, int device) {
    (void)device;
    return make_ctx(out, log_n, primes, n_q, n_p);
}

void shm_context_destroy(shm_context *ctx) {
    if (!ctx) return;
    orc_ctx_destroy(ctx->c);
    free(ctx);
}

int shm_context_info(const shm_context *ctx, uint32_t *log_n, uint32_t *n_q, uint32_t *n_p, uint32_t *dnum) {
    if (!ctx) return fail("null context");
    if (log_n) *log_n = ctx->c->log_n;
    if (n_q) *n_q = ctx->c->nq;
    if (n_p) *n_p = ctx->c->np;
    if (dnum) *dnum = ctx->dnum;
    return SHM_OK;
}

int shm_context_primes(const shm_context *ctx, uint64_t *out) {
    if (!ctx) return fail("null context");
    memcpy(out, ctx->c->primes, sizeof(uint64_t) * (ctx->c->nq + ctx->c->np));
    return SHM_OK;
}

uint32_t shm_galois_elt_from_step(const shm_context *ctx, int step) {
    return ctx ? orc_galois_elt_from_step(ctx->c->log_n, step) : 0;
}

/* ---- memory */

int shm_malloc(const shm_context *ctx, size_t bytes, void **out, void *stream) {
    (void)ctx;
    (void)stream;
    if (!out) return fail("null output pointer");
    *out = NULL;
    if (!bytes) return SHM_OK;
    if (posix_memalign(out, 64, (bytes + 63) & ~(size_t)63)) {
        *out = NULL;
        snprintf(g_err, sizeof g_err, "host allocation of %zu bytes failed", bytes);
        return SHM_ENOMEM;
    }
    return SHM_OK;
}

int shm_free(const shm_context *ctx, void *ptr, void *stream) {
    (void)ctx;
    (void)stream;
    free(ptr);
    return SHM_OK;
}

int shm_memcpy(const shm_context *ctx, void *dst, const void *src, size_t bytes, int kind, void *stream) {
    (void)ctx;
    (void)stream;
    if (kind < SHM_COPY_H2D || kind > SHM_COPY_D2D) return fail("bad copy kind");
    if (bytes) memmove(dst, src, bytes);
    return SHM_OK;
}

int shm_synchronize(const shm_context *ctx, void *stream) {
    (void)ctx;
    (void)stream;
    return SHM_OK;
}

int shm_pool_usage(const shm_context *ctx, size_t *reserved, size_t *used, size_t *used_high, int reset_high) {
    (void)ctx;
    (void)reset_high;
    if (reserved) *reserved = 0; /* host memory: not tracked */
    if (used) *used = 0;
    if (used_high) *used_high = 0;
    return SHM_OK;
}

static char g_stream_token;

int shm_stream_create(const shm_context *ctx, void **stream) {
    (void)ctx;
    if (!stream) return fail("null output pointer");
    *stream = &g_stream_token; /* host work is synchronous: any non-null token will do */
    return SHM_OK;
}

int shm_stream_destroy(const shm_context *ctx, void *stream) {
    (void)ctx;
    (void)stream;
    return SHM_OK;
}

/* CUDA graphs record device work; host arithmetic has nothing to record, so the oracle
 * refuses them (the graph tests run on the CUDA library only) */
struct shm_graph {
    int unused;
};

int shm_graph_begin(const shm_context *ctx, void *stream) {
    (void)ctx;
    (void)stream;
    return fail("CUDA graphs need the CUDA library");
}

int shm_graph_end(const shm_context *ctx, void *stream, shm_graph **out) {
    (void)ctx;
    (void)stream;
    if (out) *out = NULL;
    return fail("CUDA graphs need the CUDA library");
}

int shm_graph_launch(const shm_graph *g, void *stream) {
    (void)g;
    (void)stream;
    return fail("CUDA graphs need the CUDA library");
}

uint64_t shm_graph_kernels(const shm_graph *g) {
    (void)g;
    return 0;
}

void shm_graph_destroy(shm_graph *g) { (void)g; }

/* kernel tiles do not exist on the host: the knobs are remembered (so the host library's
 * tuning code runs unchanged) and every candidate reports zero time */
static uint32_t g_tune[2];

int shm_autotune(shm_context *ctx, int knob, uint32_t size, uint32_t level, uint32_t members, float *times,
                 uint32_t cap, uint32_t *chosen) {
    (void)ctx;
    (void)size;
    (void)level;
    (void)members;
    if (knob != SHM_TUNE_NTT_TILE && knob != SHM_TUNE_IP_CHUNK) return fail("unknown tuning knob");
    for (uint32_t i = 0; times && i < cap && i < 4; i++) times[i] = 0.0f;
    if (chosen) *chosen = g_tune[knob];
    return SHM_OK;
}

int shm_tune_get(const shm_context *ctx, int knob, uint32_t *index) {
    (void)ctx;
    if (knob != SHM_TUNE_NTT_TILE && knob != SHM_TUNE_IP_CHUNK) return fail("unknown tuning knob");
    if (!index) return fail("null output pointer");
    *index = g_tune[knob];
    return SHM_OK;
}

int shm_tune_set(shm_context *ctx, int knob, uint32_t index) {
    (void)ctx;
    if (knob != SHM_TUNE_NTT_TILE && knob != SHM_TUNE_IP_CHUNK) return fail("unknown tuning knob");
    if (index >= 4) return fail("candidate out of range");
    g_tune[knob] = index;
    return SHM_OK;
}

/* ---- sampling (same function as shmoai_b200/csrc/sampling.cu) */

static inline uint64_t mix64(uint64_t seed, uint64_t idx) {
    uint64_t z = seed + (idx + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int shm_sample_uniform(const shm_context *ctx, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t seed,
                       void *stream) {
    (void)stream;
    const orc_ctx *c = ctx->c;
    if (L < 1 || L > c->nq + c->np) return fail("level out of range");
    size_t n = c->n;
#pragma omp parallel for
    for (int row = 0; row < (int)(n_polys * L); row++) {
        uint64_t q = c->primes[row % L];
        for (size_t k = 0; k < n; k++) {
            uint64_t idx = ((uint64_t)row << c->log_n) + k;
            uint64_t h1 = mix64(seed, 2 * idx), h2 = mix64(seed, 2 * idx + 1);
            u128 t = (u128)h1 * q + (uint64_t)(((u128)h2 * q) >> 64);
            out[(size_t)row * n + k] = (uint64_t)(t >> 64);
        }
    }
    return SHM_OK;
}

int shm_sample_cbd(const shm_context *ctx, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t seed,
                   void *stream) {
    (void)stream;
    const orc_ctx *c = ctx->c;
    if (L < 1 || L > c->nq + c->np) return fail("level out of range");
    size_t n = c->n;
#pragma omp parallel for
    for (int p = 0; p < (int)n_polys; p++)
        for (size_t k = 0; k < n; k++) {
            uint64_t h = mix64(seed, ((uint64_t)p << c->log_n) + k);
            int e = __builtin_popcountll(h & 0x1FFFFFull) - __builtin_popcountll((h >> 21) & 0x1FFFFFull);
            for (uint32_t i = 0; i < L; i++) {
                uint64_t q = c->primes[i];
                out[((size_t)p * L + i) * n + k] = e >= 0 ? (uint64_t)e : q - (uint64_t)(-e);
            }
        }
    return SHM_OK;
}

/* ---- canonical-embedding encode / decode: the host encoder's FFT (radix 2, bit reversal,
 * then stages of len = 2 .. M; twiddles cos / sin (2 pi k / M), conjugated for the forward
 * transform; every product and sum rounded on its own) */

static void enc_fft(double *re, double *im, uint32_t M, int forward) {
    for (uint32_t i = 1, j = 0; i < M; i++) {
        uint32_t bit = M >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i];
            re[i] = re[j];
            re[j] = t;
            t = im[i];
            im[i] = im[j];
            im[j] = t;
        }
    }
    for (uint32_t len = 2; len <= M; len <<= 1) {
        const uint32_t stride = M / len, half = len / 2;
        for (uint32_t i = 0; i < M; i += len)
            for (uint32_t k = 0; k < half; k++) {
                const double ang = 2.0 * M_PI * (double)(k * stride) / (double)M;
                const double wr = cos(ang), wi = forward ? -sin(ang) : sin(ang);
                const double xr = re[i + k + half], xi = im[i + k + half];
                const double vr = xr * wr - xi * wi, vi = xr * wi + xi * wr;
                const double ur = re[i + k], ui = im[i + k];
                re[i + k] = ur + vr;
                im[i + k] = ui + vi;
                re[i + k + half] = ur - vr;
                im[i + k + half] = ui - vi;
            }
    }
}

static uint32_t *enc_exps(uint32_t n) {
    uint32_t M = 2 * n, slots = n / 2;
    uint32_t *e = (uint32_t *)malloc(sizeof(uint32_t) * slots);
    uint64_t v = 1;
    for (uint32_t j = 0; j < slots; j++) {
        e[j] = (uint32_t)v;
        v = (v * 5) % M;
    }
    return e;
}

size_t shm_encode_workspace_bytes(const shm_context *ctx, uint32_t n_vectors) {
    (void)ctx;
    (void)n_vectors;
    return 0;
}

int shm_encode(const shm_context *ctx, const double *re, const double *im, uint32_t n_vectors, uint32_t n_values,
               double scale, int64_t *coeffs, void *workspace, size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    const uint32_t n = ctx->c->n, M = 2 * n;
    if (n_values > n / 2) return fail("more values than slots");
    uint32_t *e = enc_exps(n);
    double *ar = (double *)malloc(sizeof(double) * M), *ai = (double *)malloc(sizeof(double) * M);
    const double f = 2.0 * scale / (double)n;
    int bad = 0;
    for (uint32_t p = 0; p < n_vectors && !bad; p++) {
        memset(ar, 0, sizeof(double) * M);
        memset(ai, 0, sizeof(double) * M);
        for (uint32_t j = 0; j < n_values; j++) {
            ar[e[j]] = re[(size_t)p * n_values + j];
            ai[e[j]] = im[(size_t)p * n_values + j];
        }
        enc_fft(ar, ai, M, 1);
        for (uint32_t k = 0; k < n; k++) {
            const double r = nearbyint(f * ar[k]);
            if (!(fabs(r) < 4611686018427387904.0)) {
                bad = 1;
                break;
            }
            coeffs[(size_t)p * n + k] = (int64_t)r;
        }
    }
    free(ar);
    free(ai);
    free(e);
    return bad ? fail("encoded values are too large") : SHM_OK;
}

int shm_decode(const shm_context *ctx, const double *coeffs, uint32_t n_vectors, double scale, double *re, double *im,
               void *workspace, size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    const uint32_t n = ctx->c->n, M = 2 * n, slots = n / 2;
    uint32_t *e = enc_exps(n);
    double *br = (double *)malloc(sizeof(double) * M), *bi = (double *)malloc(sizeof(double) * M);
    for (uint32_t p = 0; p < n_vectors; p++) {
        memset(br, 0, sizeof(double) * M);
        memset(bi, 0, sizeof(double) * M);
        for (uint32_t k = 0; k < n; k++) br[k] = coeffs[(size_t)p * n + k];
        enc_fft(br, bi, M, 0);
        for (uint32_t j = 0; j < slots; j++) {
            re[(size_t)p * slots + j] = br[e[j]] / scale;
            im[(size_t)p * slots + j] = bi[e[j]] / scale;
        }
    }
    free(br);
    free(bi);
    free(e);
    return SHM_OK;
}

int shm_lift_signed(const shm_context *ctx, const int64_t *coeffs, uint64_t *out, uint32_t n_polys, uint32_t L,
                    void *stream) {
    (void)stream;
    const orc_ctx *c = ctx->c;
    if (L < 1 || L > c->nq + c->np) return fail("level out of range");
    size_t n = c->n;
    for (uint32_t p = 0; p < n_polys; p++)
        for (uint32_t i = 0; i < L; i++)
            for (size_t k = 0; k < n; k++)
                out[((size_t)p * L + i) * n + k] = signed_residue(coeffs[(size_t)p * n + k], c->primes[i]);
    return SHM_OK;
}

/* ---- element-wise */

static int lvl_ok(const shm_context *ctx, uint32_t L) { return ctx && L >= 1 && L <= ctx->c->nq + ctx->c->np; }

int shm_ntt_forward(const shm_context *ctx, uint64_t *data, uint32_t n_polys, uint32_t L, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    orc_ntt(ctx->c, data, n_polys, L, 0);
    return SHM_OK;
}

int shm_ntt_inverse(const shm_context *ctx, uint64_t *data, uint32_t n_polys, uint32_t L, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    orc_ntt(ctx->c, data, n_polys, L, 1);
    return SHM_OK;
}

int shm_add(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys,
            uint32_t L, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    orc_add(ctx->c, a, b, out, n_polys, L);
    return SHM_OK;
}

int shm_sub(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys,
            uint32_t L, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    size_t n = ctx->c->n;
    for (size_t r = 0; r < (size_t)n_polys * L; r++) {
        uint64_t q = ctx->c->primes[r % L];
        for (size_t k = 0; k < n; k++) out[r * n + k] = submod(a[r * n + k], b[r * n + k], q);
    }
    return SHM_OK;
}

int shm_add_sizes(const shm_context *ctx, const uint64_t *a, uint32_t a_size, const uint64_t *b, uint32_t b_size,
                  uint64_t *out, uint32_t n_cts, uint32_t L, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    if (b_size > a_size || b_size == 0) return fail("add_sizes: need a_size >= b_size >= 1");
    size_t n = ctx->c->n;
    for (size_t ct = 0; ct < n_cts; ct++)
        for (size_t p = 0; p < a_size; p++)
            for (size_t l = 0; l < L; l++) {
                const uint64_t q = ctx->c->primes[l];
                const uint64_t *x = a + ((ct * a_size + p) * L + l) * n;
                uint64_t *o = out + ((ct * a_size + p) * L + l) * n;
                if (p < b_size) {
                    const uint64_t *y = b + ((ct * b_size + p) * L + l) * n;
                    for (size_t k = 0; k < n; k++) o[k] = addmod(x[k], y[k], q);
                } else {
                    memmove(o, x, n * sizeof(uint64_t));
                }
            }
    return SHM_OK;
}

int shm_negate(const shm_context *ctx, const uint64_t *a, uint64_t *out, uint32_t n_polys, uint32_t L, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    size_t n = ctx->c->n;
    for (size_t r = 0; r < (size_t)n_polys * L; r++) {
        uint64_t q = ctx->c->primes[r % L];
        for (size_t k = 0; k < n; k++) out[r * n + k] = a[r * n + k] ? q - a[r * n + k] : 0;
    }
    return SHM_OK;
}

int shm_multiply_plain(const shm_context *ctx, const uint64_t *ct, const uint64_t *pt, uint64_t *out,
                       uint32_t n_polys, uint32_t L, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    orc_multiply_plain(ctx->c, ct, pt, out, n_polys, L);
    return SHM_OK;
}

int shm_multiply(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_cts,
                 uint32_t L, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    size_t ln = (size_t)L * ctx->c->n;
    for (uint32_t i = 0; i < n_cts; i++) orc_tensor(ctx->c, a + i * 2 * ln, b + i * 2 * ln, out + i * 3 * ln, L);
    return SHM_OK;
}

int shm_permute_galois(const shm_context *ctx, const uint64_t *in, uint32_t galois_elt, uint64_t *out,
                       uint32_t n_rows, void *stream) {
    (void)stream;
    if (!ctx) return fail("null context");
    if (!(galois_elt & 1) || galois_elt >= 2 * ctx->c->n) return fail("Galois element must be odd and < 2N");
    if ((!in || !out) && n_rows) return fail("null pointer");
    if (in == out && n_rows) return fail("permute_galois cannot work in place");
    orc_apply_galois(ctx->c, in, out, n_rows, 1, galois_elt);
    return SHM_OK;
}

int shm_multiply_accumulate(const shm_context *ctx, const uint64_t *const *A, const uint64_t *const *B, uint32_t k,
                            int b_broadcast, uint64_t *out, uint32_t n_cts, uint32_t L, int accumulate, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    if (((!A || !B) && k) || (!out && n_cts)) return fail("null argument");
    size_t n = ctx->c->n, ln = (size_t)L * n;
    uint64_t *t3 = (uint64_t *)malloc(3 * ln * sizeof(uint64_t));
    if (!t3) return fail("out of host memory");
    for (uint32_t c = 0; c < n_cts; c++) {
        uint64_t *o = out + (size_t)c * 3 * ln;
        if (!accumulate) memset(o, 0, 3 * ln * sizeof(uint64_t));
        for (uint32_t t = 0; t < k; t++) {
            orc_tensor(ctx->c, A[t] + (size_t)c * 2 * ln, B[t] + (b_broadcast ? 0 : (size_t)c * 2 * ln), t3, L);
            for (uint32_t h = 0; h < 3; h++)
                for (uint32_t l = 0; l < L; l++) {
                    uint64_t q = ctx->c->primes[l], *oo = o + (h * L + l) * n, *tt = t3 + (h * L + l) * n;
                    for (size_t j = 0; j < n; j++) oo[j] = addmod(oo[j], tt[j], q);
                }
        }
    }
    free(t3);
    return SHM_OK;
}

int shm_multiply_scalar(const shm_context *ctx, const uint64_t *a, const uint64_t *scalars, uint64_t *out,
                        uint32_t n_polys, uint32_t L, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    size_t n = ctx->c->n;
    for (size_t r = 0; r < (size_t)n_polys * L; r++) {
        uint64_t q = ctx->c->primes[r % L], w = scalars[r % L];
        for (size_t k = 0; k < n; k++) out[r * n + k] = mulmod(a[r * n + k], w, q);
    }
    return SHM_OK;
}

int shm_add_scalar(const shm_context *ctx, const uint64_t *a, const uint64_t *scalars, uint64_t *out,
                   uint32_t n_cts, uint32_t L, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    size_t n = ctx->c->n, ln = (size_t)L * n;
    for (uint32_t i = 0; i < n_cts; i++) {
        const uint64_t *ai = a + i * 2 * ln;
        uint64_t *oi = out + i * 2 * ln;
        for (uint32_t j = 0; j < L; j++) {
            uint64_t q = ctx->c->primes[j];
            for (size_t k = 0; k < n; k++) oi[j * n + k] = addmod(ai[j * n + k], scalars[j], q);
        }
        memmove(oi + ln, ai + ln, ln * 8);
    }
    return SHM_OK;
}

int shm_linear_combination(const shm_context *ctx, const uint64_t *const *X, const uint32_t *X_levels,
                           const uint64_t *w, uint32_t k, const uint64_t *w0, uint64_t *out, uint32_t n_cts,
                           uint32_t L, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L) || L > 64) return fail("level out of range");
    if (!X || !X_levels || !w) return fail("null term arrays");
    if (k < 1 || k > 8) return fail("linear combination of 1..8 terms");
    for (uint32_t t = 0; t < k; t++)
        if (X_levels[t] < L) return fail("a term has fewer limbs than the result");
    const size_t n = ctx->c->n;
    for (size_t ct = 0; ct < n_cts; ct++)
        for (size_t p = 0; p < 2; p++)
            for (size_t l = 0; l < L; l++) {
                const uint64_t q = ctx->c->primes[l];
                uint64_t *o = out + ((ct * 2 + p) * L + l) * n;
                for (size_t j = 0; j < n; j++) {
                    uint64_t s = (p == 0 && w0) ? w0[l] % q : 0;
                    for (uint32_t t = 0; t < k; t++)
                        s = addmod(s, mulmod(X[t][((ct * 2 + p) * X_levels[t] + l) * n + j], w[t * L + l], q), q);
                    o[j] = s;
                }
            }
    return SHM_OK;
}

/* ---- the extended basis QlP (same semantics as the CUDA library) */

static int ks_level(const shm_context *ctx, uint32_t L);

static int ext_ok(const shm_context *ctx, uint32_t L) { return ctx && ctx->c->np && L >= 1 && L <= ctx->c->nq; }

int shm_extend(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
               void *stream) {
    (void)stream;
    if (!ext_ok(ctx, L)) return fail("level out of range");
    orc_extend(ctx->c, in, out, n_polys, L);
    return SHM_OK;
}

int shm_add_ext(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys,
                uint32_t L, void *stream) {
    (void)stream;
    if (!ext_ok(ctx, L)) return fail("level out of range");
    const orc_ctx *c = ctx->c;
    size_t n = c->n;
    uint32_t LP = L + c->np;
    for (size_t r = 0; r < (size_t)n_polys * LP; r++) {
        uint64_t q = c->primes[ext_prime(c, L, (uint32_t)(r % LP))];
        for (size_t k = 0; k < n; k++) out[r * n + k] = addmod(a[r * n + k], b[r * n + k], q);
    }
    return SHM_OK;
}

size_t shm_moddown_ext_workspace_bytes(const shm_context *ctx, uint32_t n_polys, uint32_t L) {
    (void)ctx;
    (void)n_polys;
    (void)L;
    return 0;
}

int shm_moddown_ext(const shm_context *ctx, uint64_t *ext, uint64_t *out, uint32_t n_polys, uint32_t L,
                    void *workspace, size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    if (!ext_ok(ctx, L)) return fail("level out of range");
    orc_moddown_ext(ctx->c, ext, out, n_polys, L);
    return SHM_OK;
}

int shm_multiply_plain_accumulate_ext(const shm_context *ctx, const uint64_t *const *X, const uint64_t *const *P,
                                      uint32_t k, uint64_t *out, uint32_t n_polys, uint32_t L, int accumulate,
                                      void *stream) {
    (void)stream;
    if (!ext_ok(ctx, L)) return fail("level out of range");
    const orc_ctx *c = ctx->c;
    size_t n = c->n;
    uint32_t LP = L + c->np;
#pragma omp parallel for
    for (int r = 0; r < (int)(n_polys * LP); r++) {
        uint32_t limb = (uint32_t)r % LP;
        uint64_t q = c->primes[ext_prime(c, L, limb)];
        for (size_t i = 0; i < n; i++) {
            uint64_t acc = accumulate ? out[(size_t)r * n + i] : 0;
            for (uint32_t t = 0; t < k; t++)
                acc = addmod(acc, mulmod(X[t][(size_t)r * n + i], P[t][(size_t)limb * n + i], q), q);
            out[(size_t)r * n + i] = acc;
        }
    }
    return SHM_OK;
}

int shm_lift_signed_ext(const shm_context *ctx, const int64_t *coeffs, uint64_t *out, uint32_t n_polys, uint32_t L,
                        void *stream) {
    (void)stream;
    if (!ext_ok(ctx, L)) return fail("level out of range");
    const orc_ctx *c = ctx->c;
    size_t n = c->n;
    uint32_t LP = L + c->np;
    for (uint32_t p = 0; p < n_polys; p++)
        for (uint32_t i = 0; i < LP; i++)
            for (size_t k = 0; k < n; k++)
                out[((size_t)p * LP + i) * n + k] = signed_residue(coeffs[(size_t)p * n + k], c->primes[ext_prime(c, L, i)]);
    return SHM_OK;
}

int shm_ntt_forward_ext(const shm_context *ctx, uint64_t *data, uint32_t n_polys, uint32_t L, void *stream) {
    (void)stream;
    if (!ext_ok(ctx, L)) return fail("level out of range");
    const orc_ctx *c = ctx->c;
    size_t n = c->n;
    uint32_t LP = L + c->np;
#pragma omp parallel for collapse(2)
    for (int p = 0; p < (int)n_polys; p++)
        for (int j = 0; j < (int)LP; j++) {
            uint32_t pj = ext_prime(c, L, (uint32_t)j);
            orc_ntt_fwd(data + ((size_t)p * LP + j) * n, c->log_n, c->primes[pj], c->rp + (size_t)pj * n);
        }
    return SHM_OK;
}

size_t shm_shared_rotate_ext_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                             uint32_t L) {
    (void)ctx;
    (void)n_groups;
    (void)n_members;
    (void)L;
    return 0;
}

int shm_shared_rotate_ext(const shm_context *ctx, const uint64_t *in, int in_ext, uint32_t n_groups,
                          uint32_t n_members, uint32_t n_elts, const uint32_t *elts, const uint64_t *const *keys,
                          uint64_t *const *outs, uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    if (!ks_level(ctx, L)) return fail("level out of range for key switching");
    if (!n_members) return fail("groups need at least one member");
    const orc_ctx *c = ctx->c;
    size_t n = c->n, H = n_members + 1, gin = H * (in_ext ? L + c->np : L) * n, gout = H * (L + c->np) * n;
    uint64_t **o = (uint64_t **)malloc(sizeof(uint64_t *) * (n_elts ? n_elts : 1));
    for (uint32_t g = 0; g < n_groups; g++) {
        for (uint32_t e = 0; e < n_elts; e++) o[e] = outs[e] + g * gout;
        orc_shared_rotate_ext(c, in + g * gin, in_ext, n_members, L, n_elts, elts, keys, (uint64_t *const *)o);
    }
    free(o);
    return SHM_OK;
}

int shm_multiply_plain_accumulate(const shm_context *ctx, const uint64_t *const *X, const uint64_t *const *P,
                                  uint32_t k, uint64_t *out, uint32_t n_polys, uint32_t L, int accumulate,
                                  void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L)) return fail("level out of range");
    size_t n = ctx->c->n;
#pragma omp parallel for
    for (int r = 0; r < (int)(n_polys * L); r++) {
        uint32_t limb = (uint32_t)r % L;
        uint64_t q = ctx->c->primes[limb];
        for (size_t c = 0; c < n; c++) {
            uint64_t acc = accumulate ? out[(size_t)r * n + c] : 0;
            for (uint32_t t = 0; t < k; t++)
                acc = addmod(acc, mulmod(X[t][(size_t)r * n + c], P[t][(size_t)limb * n + c], q), q);
            out[(size_t)r * n + c] = acc;
        }
    }
    return SHM_OK;
}

int shm_drop_limbs(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L_in,
                   uint32_t L_out, void *stream) {
    (void)stream;
    if (!lvl_ok(ctx, L_in) || L_out < 1 || L_out > L_in) return fail("bad limb counts");
    size_t n = ctx->c->n;
    for (uint32_t p = 0; p < n_polys; p++) memmove(out + (size_t)p * L_out * n, in + (size_t)p * L_in * n, L_out * n * 8);
    return SHM_OK;
}

/* centred lift of one-limb polynomials (mod q0, NTT form) to L limbs (NTT form) */
size_t shm_modraise_workspace_bytes(const shm_context *ctx, uint32_t n_polys) {
    (void)ctx;
    (void)n_polys;
    return 0;
}

int shm_modraise(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
                 void *workspace, size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    const orc_ctx *c = ctx->c;
    if (L < 1 || L > c->nq) return fail("level out of range");
    orc_modraise(c, in, out, n_polys, L);
    return SHM_OK;
}

/* ---- ct-pt matmul (both entry points are the same exact contraction here) */

size_t shm_ctpt_matmul_workspace_bytes(const shm_context *ctx, uint32_t n_in, uint32_t n_out, uint32_t L) {
    (void)ctx;
    (void)n_in;
    (void)n_out;
    (void)L;
    return 0;
}

int shm_ctpt_matmul_cuda_core(const shm_context *ctx, const uint64_t *X, const int64_t *W, uint64_t *Y,
                              uint32_t n_in, uint32_t n_out, uint32_t L, void *stream) {
    (void)stream;
    if (!ctx || L < 1 || L > ctx->c->nq) return fail("level out of range");
    orc_ctpt_matmul(ctx->c, X, W, n_in, n_out, L, Y);
    return SHM_OK;
}

int shm_ctpt_matmul(const shm_context *ctx, const uint64_t *X, const int64_t *W, uint64_t *Y, uint32_t n_in,
                    uint32_t n_out, uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    return shm_ctpt_matmul_cuda_core(ctx, X, W, Y, n_in, n_out, L, stream);
}

/* ---- level and key switching */

size_t shm_rescale_workspace_bytes(const shm_context *ctx, uint32_t n_polys, uint32_t L) {
    (void)ctx;
    (void)n_polys;
    (void)L;
    return 0;
}

int shm_rescale(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
                void *workspace, size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    if (!ctx || L < 2 || L > ctx->c->nq) return fail("rescale needs 2 <= L <= n_q limbs");
    orc_rescale(ctx->c, in, out, n_polys, L);
    return SHM_OK;
}

static int ks_level(const shm_context *ctx, uint32_t L) {
    const orc_ctx *c = ctx->c;
    return L >= 1 && L <= c->nq && c->np && (L + c->np - 1) / c->np <= ctx->dnum;
}

size_t shm_keyswitch_workspace_bytes(const shm_context *ctx, uint32_t n_cts, uint32_t L) {
    (void)ctx;
    (void)n_cts;
    (void)L;
    return 0;
}

int shm_relinearize(const shm_context *ctx, const uint64_t *ct3, const uint64_t *relin_key, uint64_t *out,
                    uint32_t n_cts, uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    if (!ks_level(ctx, L)) return fail("level out of range for key switching");
    size_t ln = (size_t)L * ctx->c->n;
    for (uint32_t i = 0; i < n_cts; i++) orc_relinearize(ctx->c, ct3 + i * 3 * ln, L, relin_key, ctx->dnum, out + i * 2 * ln);
    return SHM_OK;
}

int shm_relinearize_rescale(const shm_context *ctx, const uint64_t *ct3, const uint64_t *relin_key, uint64_t *out,
                            uint32_t n_cts, uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    if (!ks_level(ctx, L) || L < 2) return fail("relinearize-rescale needs 2 <= L <= n_q");
    if (!ct3 || !relin_key || !out) return fail("null argument");
    size_t ln = (size_t)L * ctx->c->n;
    const uint64_t *ae = ct3 + (size_t)n_cts * 3 * ln, *oe = out + (size_t)n_cts * 2 * (ln - ctx->c->n);
    if (n_cts && (const uint64_t *)out < ae && ct3 < oe) return fail("relinearize-rescale output overlaps its input");
    for (uint32_t i = 0; i < n_cts; i++)
        orc_relin_rescale(ctx->c, ct3 + i * 3 * ln, L, relin_key, out + (size_t)i * 2 * (ln - ctx->c->n));
    return SHM_OK;
}

int shm_apply_galois(const shm_context *ctx, const uint64_t *ct, uint32_t galois_elt, const uint64_t *galois_key,
                     uint64_t *out, uint32_t n_cts, uint32_t L, void *workspace, size_t workspace_bytes,
                     void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    if (!ks_level(ctx, L)) return fail("level out of range for key switching");
    if (!(galois_elt & 1) || galois_elt >= 2 * ctx->c->n) return fail("Galois element must be odd and < 2N");
    size_t ln = (size_t)L * ctx->c->n;
    for (uint32_t i = 0; i < n_cts; i++)
        orc_apply_galois_ct(ctx->c, ct + i * 2 * ln, L, galois_elt, galois_key, ctx->dnum, out + i * 2 * ln);
    return SHM_OK;
}

size_t shm_apply_galois_hoisted_workspace_bytes(const shm_context *ctx, uint32_t n_cts, uint32_t L) {
    (void)ctx;
    (void)n_cts;
    (void)L;
    return 0;
}

int shm_apply_galois_hoisted(const shm_context *ctx, const uint64_t *ct, uint32_t n_elts, const uint32_t *elts,
                             const uint64_t *const *keys, uint64_t *const *outs, uint32_t n_cts, uint32_t L,
                             void *workspace, size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    if (!ks_level(ctx, L)) return fail("level out of range for key switching");
    size_t ln = (size_t)L * ctx->c->n;
    uint64_t **o = (uint64_t **)malloc(sizeof(uint64_t *) * (n_elts ? n_elts : 1));
    for (uint32_t i = 0; i < n_cts; i++) {
        for (uint32_t e = 0; e < n_elts; e++) o[e] = outs[e] + i * 2 * ln;
        orc_apply_galois_hoisted(ctx->c, ct + i * 2 * ln, L, n_elts, elts, keys, ctx->dnum, (uint64_t *const *)o);
    }
    free(o);
    return SHM_OK;
}

size_t shm_shared_rotate_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members, uint32_t L) {
    (void)ctx;
    (void)n_groups;
    (void)n_members;
    (void)L;
    return 0;
}

size_t shm_shared_rotate_one_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                             uint32_t L) {
    (void)ctx;
    (void)n_groups;
    (void)n_members;
    (void)L;
    return 0;
}

/* the reference's order (ShRotate.cu:218-256): the automorphism on every row, then the
 * hoisted key switch with the identity element */
int shm_shared_rotate(const shm_context *ctx, const uint64_t *sh, uint32_t n_groups, uint32_t n_members, uint32_t elt,
                      const uint64_t *key, uint64_t *out, uint32_t L, void *workspace, size_t workspace_bytes,
                      void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    if (!ks_level(ctx, L)) return fail("level out of range for key switching");
    if (!key || !out || !n_members || out == sh) return fail("bad shared-a rotation arguments");
    if (elt % 2 == 0 || elt >= 2 * ctx->c->n) return fail("Galois element must be odd and below 2N");
    size_t gl = (size_t)(n_members + 1) * L * ctx->c->n;
    uint64_t *rot = (uint64_t *)malloc(gl * 8);
    const uint32_t one = 1;
    const uint64_t *k = key;
    for (uint32_t g = 0; g < n_groups; g++) {
        orc_apply_galois(ctx->c, sh + g * gl, rot, n_members + 1, L, elt);
        uint64_t *o = out + g * gl;
        orc_shared_rotate_hoisted(ctx->c, rot, n_members, L, 1, &one, &k, (uint64_t *const *)&o);
    }
    free(rot);
    return SHM_OK;
}

int shm_shared_rotate_hoisted(const shm_context *ctx, const uint64_t *sh, uint32_t n_groups, uint32_t n_members,
                              uint32_t n_elts, const uint32_t *elts, const uint64_t *const *keys, uint64_t *const *outs,
                              uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    if (!ks_level(ctx, L)) return fail("level out of range for key switching");
    size_t gl = (size_t)(n_members + 1) * L * ctx->c->n;
    uint64_t **o = (uint64_t **)malloc(sizeof(uint64_t *) * (n_elts ? n_elts : 1));
    for (uint32_t g = 0; g < n_groups; g++) {
        for (uint32_t e = 0; e < n_elts; e++) o[e] = outs[e] + g * gl;
        orc_shared_rotate_hoisted(ctx->c, sh + g * gl, n_members, L, n_elts, elts, keys, (uint64_t *const *)o);
    }
    free(o);
    return SHM_OK;
}

size_t shm_fmt_switch_forward_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                              uint32_t L) {
    (void)ctx;
    (void)n_groups;
    (void)n_members;
    (void)L;
    return 0;
}

int shm_fmt_switch_forward(const shm_context *ctx, const uint64_t *cts, uint32_t n_groups, uint32_t n_members,
                           const uint64_t *key, uint64_t *out, uint32_t L, void *workspace, size_t workspace_bytes,
                           void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    if (!ctx || L < 1 || L > ctx->c->nq) return fail("level out of range");
    size_t ln = (size_t)L * ctx->c->n;
    for (uint32_t g = 0; g < n_groups; g++)
        orc_fmt_forward(ctx->c, cts + (size_t)g * n_members * 2 * ln, n_members, L, key,
                        out + (size_t)g * (n_members + 1) * ln);
    return SHM_OK;
}

size_t shm_fmt_switch_backward_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                               uint32_t L) {
    (void)ctx;
    (void)n_groups;
    (void)n_members;
    (void)L;
    return 0;
}

int shm_fmt_switch_backward(const shm_context *ctx, const uint64_t *sh, uint32_t n_groups, uint32_t n_members,
                            const uint64_t *const *keys, uint64_t *out, uint32_t L, void *workspace,
                            size_t workspace_bytes, void *stream) {
    (void)workspace;
    (void)workspace_bytes;
    (void)stream;
    if (!ks_level(ctx, L)) return fail("level out of range for key switching");
    size_t ln = (size_t)L * ctx->c->n;
    for (uint32_t g = 0; g < n_groups; g++)
        orc_fmt_backward(ctx->c, sh + (size_t)g * (n_members + 1) * ln, n_members, L, keys,
                         out + (size_t)g * n_members * 2 * ln);
    return SHM_OK;
}
