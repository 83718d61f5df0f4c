// Context construction and the extern "C" entry points of include/shmoai_ckks.h.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/shmoai_ckks.h"
#include "core.hpp"
#include "host_math.hpp"

namespace shm {

std::atomic<unsigned long long> g_launches{0};

namespace {

template <typename T>
T *upload(const std::vector<T> &v) {
    T *d = nullptr;
    SHM_CUDA(cudaMalloc(&d, v.size() * sizeof(T)));
    SHM_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}

void push4(std::vector<uint64_t> &v, uint64_t c, uint64_t psi_half_inv, uint64_t q) {
    uint64_t c1 = host::mulmod(c, psi_half_inv, q);
    v.push_back(c);
    v.push_back(host::shoup_of(c, q));
    v.push_back(c1);
    v.push_back(host::shoup_of(c1, q));
}

}  // namespace

Context::~Context() {
    cudaSetDevice(device);
    release_encode_tables(*this);
    for (void *p : {(void *)pc, (void *)tw, (void *)twq, (void *)inv_scale_plain, (void *)moddown_scale, (void *)moddown_conv,
                    (void *)p_inv, (void *)p_mod, (void *)rescale_inv, arena})
        if (p) cudaFree(p);
    for (auto &l : ks)
        for (void *p : {(void *)l.modup_scale, (void *)l.modup_conv, (void *)l.rr_scale, (void *)l.rr_conv,
                        (void *)l.rr_sinv, (void *)l.rr_vs, (void *)l.rr_inv_s})
            if (p) cudaFree(p);
    for (auto &kv : galois_perm) cudaFree(kv.second);
    for (auto &kv : ext_consts)
        for (void *p : kv.second) cudaFree(p);
    if (pool) {
        cudaDeviceSynchronize();
        cudaMemPoolDestroy(pool);
    }
    (void)cudaGetLastError();  // the frees above report nothing a caller could act on
}

cudaMemPool_t Context::mempool() {
    std::lock_guard<std::mutex> g(mu);
    if (!pool) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        SHM_CUDA(cudaMemPoolCreate(&pool, &props));
        uint64_t keep = ~0ull;  // never return freed blocks to the driver on synchronisation
        SHM_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    return pool;
}

__global__ void perm_table_kernel(uint32_t *p, uint32_t elt, uint32_t log_n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    p[k] = galois_index(k, elt, log_n);
}

const uint32_t *Context::perm(uint32_t elt) {
    std::lock_guard<std::mutex> g(mu);
    auto it = galois_perm.find(elt);
    if (it != galois_perm.end()) return it->second;
    if (!(elt & 1) || elt >= 2 * n) throw std::invalid_argument("Galois element must be odd and < 2N");
    // NTT-domain automorphism (src/galois.cu:8-21, include/galois.cuh:44-60):
    // slot k holds a(psi^(2*brv(k)+1)); X -> X^elt moves slot perm[k] to k with
    // 2*brv(perm[k]) + 1 = (2*brv(k) + 1) * elt mod 2N.
    // built on the device (the table of galois_index), then waited for once: every stream may use it
    uint32_t *d = nullptr;
    SHM_CUDA(cudaMalloc(&d, (size_t)n * sizeof(uint32_t)));
    perm_table_kernel<<<n / 256, 256>>>(d, elt, log_n);
    SHM_CUDA(cudaGetLastError());
    SHM_CUDA(cudaStreamSynchronize(0));
    galois_perm[elt] = d;
    return d;
}

void *Context::workspace(size_t bytes) {
    if (bytes <= arena_bytes) return arena;
    if (arena) SHM_CUDA(cudaFree(arena));
    arena = nullptr;
    arena_bytes = 0;
    SHM_CUDA(cudaMalloc(&arena, bytes));
    arena_bytes = bytes;
    return arena;
}

Context *create_context(uint32_t log_n, const std::vector<uint64_t> &primes, uint32_t nq, uint32_t np, int device) {
    if (log_n != 12 && log_n != 16) throw std::invalid_argument("log_n must be 12 or 16");
    if (nq < 1 || nq + np != primes.size() || nq + np > 250) throw std::invalid_argument("bad prime counts");
    std::unique_ptr<Context> c(new Context);
    c->device = device;
    SHM_CUDA(cudaSetDevice(device));
    c->log_n = log_n;
    c->n = 1u << log_n;
    c->nq = nq;
    c->np = np;
    c->dnum = np ? nq / np : 0;
    c->primes = primes;
    const uint32_t QP = nq + np, n = c->n;
    for (uint64_t q : primes) {
        if (q >= (1ull << 61) || (q - 1) % (2ull * n) || !host::is_prime(q))
            throw std::invalid_argument("every prime must be < 2^61 and 1 mod 2N");
        if (np && (uint64_t)np * q >= (1ull << 63))
            throw std::invalid_argument("alpha * q must stay below 2^63 for the lazy base conversion");
    }
    c->s52 = *std::max_element(primes.begin(), primes.end()) < kS52PrimeLimit;
    {
        int fam = 0;
        for (uint64_t q : primes) fam |= (1 << bf_mode_of(q)) | (1 << fwd_mode_of(q));
        c->ntt_families = (fam & ~kFamSmall) == 0 ? kFamSmall : (fam & ~kFamLarge) == 0 ? kFamLarge : kFamAll;
    }
    // per-prime constants and twiddles
    std::vector<uint64_t> tw((size_t)QP * 4 * n), psi_half_inv(QP), sc_plain;
    for (uint32_t i = 0; i < QP; i++) {
        uint64_t q = primes[i], *t = tw.data() + (size_t)i * 4 * n;
        host::ntt_tables(q, log_n, t, t + n, t + 2 * n, t + 3 * n);
        psi_half_inv[i] = t[2 * n + 1];
        PrimeConst p{};
        p.q = q;
        p.mu = host::barrett_mu(q);
        p.shift = host::bit_length(q) - 1;
        {
            const uint32_t k = p.shift + 1, s = k > 25 ? k - 25 : 0;
            p.red_m = (uint32_t)(((unsigned __int128)1 << (32 + s)) / q);
        }
        p.n_inv = host::invmod(n, q);
        p.n_inv_shoup = host::shoup_of(p.n_inv, q);
        c->h_pc.push_back(p);
        push4(sc_plain, p.n_inv, psi_half_inv[i], q);
    }
    c->pc = upload(c->h_pc);
    c->tw = upload(tw);
    {
        // for the FP64 butterflies of the primes below kF64CentreLimit (other primes never read it):
        // the forward and inverse w / q rounded to the nearest double (w and q are exact doubles
        // below 2^53), then the forward w itself as a double.  The forward twiddles of the primes
        // at or above kF64GrowLimit (the centred family) are kept within q/2 of zero (w - q for
        // w > q/2), so that |w / q| <= 1/2.
        std::vector<double> twq((size_t)QP * 3 * n, 0.0);
        for (uint32_t i = 0; i < QP; i++) {
            if (primes[i] >= kF64CentreLimit) continue;
            const uint64_t q = primes[i];
            const double qd = (double)q;
            const bool centre = q >= kF64GrowLimit;
            const uint64_t *t = tw.data() + (size_t)i * 4 * n;
            double *d = twq.data() + (size_t)i * 3 * n;
            for (uint32_t k = 0; k < n; k++) {
                const double w = centre && t[k] > q / 2 ? (double)t[k] - qd : (double)t[k];
                d[k] = w / qd;
                d[n + k] = (double)t[2 * n + k] / qd;
                d[2 * n + k] = w;
            }
        }
        c->twq = upload(twq);
    }
    c->inv_scale_plain = upload(sc_plain);

    // rescale: row L-1 holds q_{L-1}^-1 mod q_j
    std::vector<uint64_t> rinv((size_t)nq * nq * 2, 0);
    for (uint32_t L = 2; L <= nq; L++)
        for (uint32_t j = 0; j + 1 < L; j++) {
            uint64_t q = primes[j], v = host::invmod(primes[L - 1] % q, q);
            rinv[((size_t)(L - 1) * nq + j) * 2] = v;
            rinv[((size_t)(L - 1) * nq + j) * 2 + 1] = host::shoup_of(v, q);
        }
    c->rescale_inv = upload(rinv);

    c->ks.resize(nq + 1);
    if (np) {
        std::vector<uint64_t> P(primes.begin() + nq, primes.end());
        // ModDown constants
        std::vector<uint64_t> mds, mdc((size_t)nq * np), pinv((size_t)nq * 2);
        for (uint32_t k = 0; k < np; k++) {
            uint64_t p = P[k], h = host::partial_product(P, k, p);
            push4(mds, host::mulmod(host::invmod(h, p), c->h_pc[nq + k].n_inv, p), psi_half_inv[nq + k], p);
        }
        for (uint32_t j = 0; j < nq; j++) {
            uint64_t q = primes[j], prod = 1;
            for (uint32_t k = 0; k < np; k++) {
                mdc[(size_t)j * np + k] = host::partial_product(P, k, q);
                prod = host::mulmod(prod, P[k] % q, q);
            }
            uint64_t v = host::invmod(prod, q);
            pinv[2 * j] = v;
            pinv[2 * j + 1] = host::shoup_of(v, q);
        }
        std::vector<uint64_t> pmod((size_t)nq * 2);
        for (uint32_t j = 0; j < nq; j++) {
            uint64_t q = primes[j], prod = 1;
            for (uint32_t k = 0; k < np; k++) prod = host::mulmod(prod, P[k] % q, q);
            pmod[2 * j] = prod;
            pmod[2 * j + 1] = host::shoup_of(prod, q);
        }
        c->moddown_scale = upload(mds);
        c->moddown_conv = upload(mdc);
        c->p_inv = upload(pinv);
        c->p_mod = upload(pmod);
        c->h_p_mod = pmod;
        // ModUp constants per level
        for (uint32_t L = 1; L <= nq; L++) {
            LevelKS &ks = c->ks[L];
            ks.L = L;
            ks.beta = (L + np - 1) / np;
            const uint32_t LP = L + np;
            std::vector<uint64_t> msc, conv((size_t)ks.beta * LP * np, 0);
            for (uint32_t b = 0; b < ks.beta; b++) {
                uint32_t s = b * np, e = std::min(s + np, L);
                std::vector<uint64_t> D(primes.begin() + s, primes.begin() + e);
                for (uint32_t i = s; i < e; i++) {
                    uint64_t q = primes[i], h = host::partial_product(D, i - s, q);
                    push4(msc, host::mulmod(host::invmod(h, q), c->h_pc[i].n_inv, q), psi_half_inv[i], q);
                }
                for (uint32_t j = 0; j < LP; j++) {
                    if (j >= s && j < e) continue;
                    uint64_t t = primes[j < L ? j : nq + (j - L)];
                    for (uint32_t i = 0; i < e - s; i++)
                        conv[((size_t)b * LP + j) * np + i] = host::partial_product(D, i, t);
                }
            }
            ks.modup_scale = upload(msc);
            ks.modup_conv = upload(conv);
            if (L < 2) continue;
            // ModDown by S = q_{L-1} P
            std::vector<uint64_t> S{primes[L - 1]};
            std::vector<uint32_t> sidx{L - 1};
            for (uint32_t k = 0; k < np; k++) {
                S.push_back(P[k]);
                sidx.push_back(nq + k);
            }
            std::vector<uint64_t> rsc, rconv((size_t)(L - 1) * (np + 1)), rsinv((size_t)(L - 1) * 2);
            for (uint32_t k = 0; k <= np; k++) {
                const uint64_t s = S[k], h = host::partial_product(S, k, s);
                push4(rsc, host::mulmod(host::invmod(h, s), c->h_pc[sidx[k]].n_inv, s), psi_half_inv[sidx[k]], s);
            }
            for (uint32_t j = 0; j + 1 < L; j++) {
                const uint64_t q = primes[j];
                uint64_t prod = 1;
                for (uint32_t k = 0; k <= np; k++) {
                    rconv[(size_t)j * (np + 1) + k] = host::partial_product(S, k, q);
                    prod = host::mulmod(prod, S[k] % q, q);
                }
                const uint64_t v = host::invmod(prod, q);
                rsinv[2 * j] = v;
                rsinv[2 * j + 1] = host::shoup_of(v, q);
            }
            std::vector<uint64_t> rvs((size_t)(L - 1) * 16);
            for (uint32_t j = 0; j + 1 < L; j++) {
                const uint64_t q = primes[j];
                uint64_t Sq = 1;
                for (uint32_t k = 0; k <= np; k++) Sq = host::mulmod(Sq, S[k] % q, q);
                for (uint32_t v = 0; v < 16; v++) rvs[(size_t)j * 16 + v] = host::mulmod(v, Sq, q);
            }
            std::vector<double> rinvs(np + 1);
            for (uint32_t k = 0; k <= np; k++) rinvs[k] = 1.0 / (double)S[k];
            ks.rr_scale = upload(rsc);
            ks.rr_conv = upload(rconv);
            ks.rr_sinv = upload(rsinv);
            ks.rr_vs = upload(rvs);
            ks.rr_inv_s = upload(rinvs);
        }
    }
    SHM_CUDA(cudaDeviceSynchronize());
    return c.release();
}

}  // namespace shm

// ---------------------------------------------------------------------------
// C ABI

struct shm_context {
    shm::Context *c;
};

namespace {

thread_local std::string g_err;

template <typename F>
int guard(F &&f) {
    // the runtime's last-error slot may hold a non-sticky error left by a call outside this library
    // (or ignored in a destructor); it is not this call's, so it is cleared before the call's own
    // launch checks read the slot.  Sticky errors (a faulted context) survive this and still fail.
    (void)cudaGetLastError();
    try {
        f();
        return SHM_OK;
    } catch (const std::invalid_argument &e) {
        g_err = e.what();
        return SHM_EINVAL;
    } catch (const shm::CudaError &e) {
        g_err = e.what();
        return std::strstr(e.what(), "out of memory") ? SHM_ENOMEM : SHM_ECUDA;
    } catch (const std::exception &e) {
        g_err = e.what();
        return SHM_EINTERNAL;
    } catch (...) {
        g_err = "unknown error";
        return SHM_EINTERNAL;
    }
}

shm::Context &ctx_of(const shm_context *h) {
    if (!h || !h->c) throw std::invalid_argument("null context");
    return *h->c;
}

cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Element-wise operations and NTTs accept key-level polynomials (all nq + np primes);
// level-changing operations check L <= nq themselves.
void check_level(const shm::Context &c, uint32_t L) {
    if (L < 1 || L > c.nq + c.np) throw std::invalid_argument("level (limb count) out of range");
}

uint64_t *ws_of(shm::Context &c, void *ws, size_t have, size_t need_words) {
    size_t need = need_words * 8;
    if (ws) {
        if (have < need) throw std::invalid_argument("workspace too small");
        return static_cast<uint64_t *>(ws);
    }
    return static_cast<uint64_t *>(c.workspace(need));
}

void set_device(const shm::Context &c) { SHM_CUDA(cudaSetDevice(c.device)); }

}  // namespace

extern "C" {

const char *shm_last_error(void) { return g_err.c_str(); }

uint64_t shm_kernel_launches(void) { return shm::g_launches.load(std::memory_order_relaxed); }

int shm_context_create_from_primes(shm_context **out, uint32_t log_n, const uint64_t *primes, uint32_t n_q,
                                   uint32_t n_p, int device) {
    return guard([&] {
        if (!out || !primes) throw std::invalid_argument("null argument");
        std::vector<uint64_t> p(primes, primes + n_q + n_p);
        *out = new shm_context{shm::create_context(log_n, p, n_q, n_p, device)};
    });
}

int shm_context_create(shm_context **out, uint32_t log_n, const int *bits, uint32_t n_q, uint32_t n_p, int device) {
    return guard([&] {
        if (!out || !bits) throw std::invalid_argument("null argument");
        std::vector<int> b(bits, bits + n_q + n_p);
        auto p = shm::host::create_primes((int)log_n, b);
        *out = new shm_context{shm::create_context(log_n, p, n_q, n_p, device)};
    });
}

void shm_context_destroy(shm_context *ctx) {
    if (!ctx) return;
    delete ctx->c;
    delete ctx;
}

int shm_context_info(const shm_context *ctx, uint32_t *log_n, uint32_t *n_q, uint32_t *n_p, uint32_t *dnum) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        if (log_n) *log_n = c.log_n;
        if (n_q) *n_q = c.nq;
        if (n_p) *n_p = c.np;
        if (dnum) *dnum = c.dnum;
    });
}

int shm_context_primes(const shm_context *ctx, uint64_t *out) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        std::memcpy(out, c.primes.data(), c.primes.size() * sizeof(uint64_t));
    });
}

int shm_ntt_forward(const shm_context *ctx, uint64_t *data, uint32_t n_polys, uint32_t L, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        set_device(c);
        shm::ntt_forward(c, data, n_polys * L, L, shm::q_map(L), S(stream));
    });
}

int shm_ntt_inverse(const shm_context *ctx, uint64_t *data, uint32_t n_polys, uint32_t L, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        set_device(c);
        shm::ntt_inverse(c, data, n_polys * L, L, shm::q_map(L), nullptr, S(stream));
    });
}

static int ew(const shm_context *ctx, shm::EwOp op, const uint64_t *a, const uint64_t *b, uint64_t *out,
              uint32_t n_polys, uint32_t L, uint32_t b_polys, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        set_device(c);
        shm::elementwise(c, op, a, b, out, n_polys, L, b_polys, S(stream));
    });
}

int shm_add(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys,
            uint32_t L, void *stream) {
    return ew(ctx, shm::EwOp::Add, a, b, out, n_polys, L, n_polys, stream);
}

int shm_sub(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys,
            uint32_t L, void *stream) {
    return ew(ctx, shm::EwOp::Sub, a, b, out, n_polys, L, n_polys, stream);
}

int shm_add_sizes(const shm_context *ctx, const uint64_t *a, uint32_t a_size, const uint64_t *b, uint32_t b_size,
                  uint64_t *out, uint32_t n_cts, uint32_t L, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        set_device(c);
        shm::add_sizes(c, a, a_size, b, b_size, out, n_cts, L, S(stream));
    });
}

int shm_negate(const shm_context *ctx, const uint64_t *a, uint64_t *out, uint32_t n_polys, uint32_t L, void *stream) {
    return ew(ctx, shm::EwOp::Negate, a, nullptr, out, n_polys, L, n_polys, stream);
}

int shm_multiply_plain(const shm_context *ctx, const uint64_t *ct, const uint64_t *pt, uint64_t *out,
                       uint32_t n_polys, uint32_t L, void *stream) {
    return ew(ctx, shm::EwOp::MulPlain, ct, pt, out, n_polys, L, 1, stream);
}

int shm_multiply(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_cts,
                 uint32_t L, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        set_device(c);
        shm::tensor(c, a, b, out, n_cts, L, S(stream));
    });
}

int shm_permute_galois(const shm_context *ctx, const uint64_t *in, uint32_t galois_elt, uint64_t *out,
                       uint32_t n_rows, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        if (!(galois_elt & 1) || galois_elt >= 2 * c.n) throw std::invalid_argument("Galois element must be odd and < 2N");
        if ((!in || !out) && n_rows) throw std::invalid_argument("null pointer");
        if (in == out && n_rows) throw std::invalid_argument("permute_galois cannot work in place");
        set_device(c);
        shm::apply_galois(c, in, out, n_rows, galois_elt, S(stream));
    });
}

int shm_multiply_accumulate(const shm_context *ctx, const uint64_t *const *A, const uint64_t *const *B, uint32_t k,
                            int b_broadcast, uint64_t *out, uint32_t n_cts, uint32_t L, int accumulate, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        if ((!A || !B) && k) throw std::invalid_argument("null term arrays");
        if (!out && n_cts) throw std::invalid_argument("null output");
        set_device(c);
        // 2 * chunk products (the middle term) must stay below the Barrett bound 2^(63 + bits(q))
        uint32_t chunk = shm::kMaxAccTerms;
        for (uint32_t i = 0; i < L; i++) {
            const int b = shm::host::bit_length(c.primes[i]);
            const int room = 63 + b - 2 * b;  // log2 of the products one sum may hold
            const uint32_t lim = room >= 6 ? 64u : (1u << room);
            chunk = std::min(chunk, std::max(1u, lim / 2));
        }
        for (uint32_t t0 = 0; t0 < k; t0 += chunk) {
            const uint32_t kk = std::min(chunk, k - t0);
            shm::PtrTab a{}, b{};
            for (uint32_t t = 0; t < kk; t++) {
                if (!A[t0 + t] || !B[t0 + t]) throw std::invalid_argument("null term");
                a.p[t] = A[t0 + t];
                b.p[t] = B[t0 + t];
            }
            shm::tensor_accumulate(c, a, b, kk, 1, b_broadcast ? 0 : 1, out, n_cts, L, accumulate || t0 > 0,
                                   S(stream));
        }
        if (k == 0 && !accumulate && n_cts)
            SHM_CUDA(cudaMemsetAsync(out, 0, (size_t)n_cts * 3 * L * c.n * 8, S(stream)));
    });
}

size_t shm_rescale_workspace_bytes(const shm_context *ctx, uint32_t n_polys, uint32_t L) {
    return ctx && ctx->c ? shm::rescale_ws_words(*ctx->c, n_polys, L) * 8 : 0;
}

int shm_rescale(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
                void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        if (L < 2 || L > c.nq) throw std::invalid_argument("rescale needs 2 <= L <= n_q limbs");
        set_device(c);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, shm::rescale_ws_words(c, n_polys, L));
        shm::rescale(c, in, out, n_polys, L, ws, S(stream));
    });
}

size_t shm_keyswitch_workspace_bytes(const shm_context *ctx, uint32_t n_cts, uint32_t L) {
    return ctx && ctx->c ? shm::keyswitch_ws_words(*ctx->c, n_cts, L) * 8 : 0;
}

int shm_keyswitch(const shm_context *ctx, const uint64_t *d, const uint64_t *key, uint64_t *out, uint32_t n_cts,
                  uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        set_device(c);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, shm::keyswitch_ws_words(c, n_cts, L));
        const size_t ln = (size_t)L * c.n;
        shm::KsOutput o{out, out + ln, nullptr, nullptr, 2 * ln};
        shm::keyswitch(c, d, ln, n_cts, L, key, o, ws, S(stream));
    });
}

int shm_relinearize(const shm_context *ctx, const uint64_t *ct3, const uint64_t *relin_key, uint64_t *out,
                    uint32_t n_cts, uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        set_device(c);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, shm::keyswitch_ws_words(c, n_cts, L));
        const size_t ln = (size_t)L * c.n;
        if (out == ct3 && n_cts > 1) throw std::invalid_argument("in-place relinearize needs n_cts == 1");
        // key switch c2 first (it only reads ct3), then out_h = c_h + cx_h in the combine step;
        // (c0, c1) are read with the size-3 stride through the add pointers
        shm::KsOutput o{out, out + ln, ct3, ct3 + ln, 2 * ln};
        if (out != ct3) {
            // the combine reads add and writes out with one stride: stage (c0, c1) into out
            SHM_CUDA(cudaMemcpy2DAsync(out, 2 * ln * 8, ct3, 3 * ln * 8, 2 * ln * 8, n_cts,
                                       cudaMemcpyDeviceToDevice, S(stream)));
            o.add0 = out;
            o.add1 = out + ln;
        }
        shm::keyswitch(c, ct3 + 2 * ln, 3 * ln, n_cts, L, relin_key, o, ws, S(stream));
    });
}

int shm_relinearize_rescale(const shm_context *ctx, const uint64_t *ct3, const uint64_t *relin_key, uint64_t *out,
                            uint32_t n_cts, uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        set_device(c);
        if (!ct3 || !relin_key || !out) throw std::invalid_argument("null argument");
        const size_t ln = (size_t)L * c.n;
        const uint64_t *a = ct3, *ae = ct3 + (size_t)n_cts * 3 * ln;
        const uint64_t *o = out, *oe = out + (size_t)n_cts * 2 * (ln - c.n);
        if (n_cts && o < ae && a < oe) throw std::invalid_argument("relinearize-rescale output overlaps its input");
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, shm::keyswitch_ws_words(c, n_cts, L));
        shm::relin_rescale(c, ct3, n_cts, L, relin_key, out, ws, S(stream));
    });
}

uint32_t shm_galois_elt_from_step(const shm_context *ctx, int step) {
    if (!ctx || !ctx->c) return 0;
    const uint32_t n = ctx->c->n;
    const uint64_t m = 2ull * n;
    if (step == 0) return (uint32_t)(m - 1);
    // left rotation by |step| slots uses 5^step; right rotation by s uses 5^(N/2 - s)
    uint32_t pos = (uint32_t)(step < 0 ? -step : step);
    if (pos >= n / 2) return 0;
    uint32_t e = step < 0 ? n / 2 - pos : pos;
    uint64_t g = 1;
    while (e--) g = (g * 5) & (m - 1);
    return (uint32_t)g;
}

int shm_apply_galois(const shm_context *ctx, const uint64_t *ct, uint32_t galois_elt, const uint64_t *galois_key,
                     uint64_t *out, uint32_t n_cts, uint32_t L, void *workspace, size_t workspace_bytes,
                     void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        set_device(c);
        const size_t ln = (size_t)L * c.n;
        const size_t ks_words = shm::keyswitch_ws_words(c, n_cts, L);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, ks_words + (size_t)n_cts * 2 * ln);
        uint64_t *perm = ws + ks_words;  // permuted (c0, c1) of every ciphertext
        shm::apply_galois(c, ct, perm, n_cts * 2 * L, galois_elt, S(stream));
        shm::KsOutput o{out, out + ln, perm, nullptr, 2 * ln};
        shm::keyswitch(c, perm + ln, 2 * ln, n_cts, L, galois_key, o, ws, S(stream));
    });
}

size_t shm_apply_galois_hoisted_workspace_bytes(const shm_context *ctx, uint32_t n_cts, uint32_t L) {
    return ctx && ctx->c ? shm::hoisted_ws_words(*ctx->c, n_cts, L) * 8 : 0;
}

int shm_apply_galois_hoisted(const shm_context *ctx, const uint64_t *ct, uint32_t n_elts, const uint32_t *elts,
                             const uint64_t *const *keys, uint64_t *const *outs, uint32_t n_cts, uint32_t L,
                             void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        if (!elts || !keys || !outs) throw std::invalid_argument("null element, key or output array");
        for (uint32_t e = 0; e < n_elts; e++)
            if (outs[e] == ct) throw std::invalid_argument("hoisted outputs must not alias the input");
        set_device(c);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, shm::hoisted_ws_words(c, n_cts, L));
        shm::apply_galois_hoisted(c, ct, n_cts, L, n_elts, elts, keys, outs, ws, S(stream));
    });
}

size_t shm_shared_rotate_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members, uint32_t L) {
    return ctx && ctx->c ? shm::shared_rotate_ws_words(*ctx->c, n_groups, n_members, L) * 8 : 0;
}

int shm_shared_rotate_hoisted(const shm_context *ctx, const uint64_t *sh, uint32_t n_groups, uint32_t n_members,
                              uint32_t n_elts, const uint32_t *elts, const uint64_t *const *keys, uint64_t *const *outs,
                              uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        if (!elts || !keys || !outs || n_members == 0) throw std::invalid_argument("bad shared-a rotation arguments");
        for (uint32_t e = 0; e < n_elts; e++)
            if (outs[e] == sh) throw std::invalid_argument("outputs must not alias the input");
        set_device(c);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, shm::shared_rotate_ws_words(c, n_groups, n_members, L));
        shm::shared_rotate_hoisted(c, sh, n_groups, n_members, L, n_elts, elts, keys, outs, ws, S(stream));
    });
}

size_t shm_shared_rotate_one_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                             uint32_t L) {
    if (!ctx || !ctx->c) return 0;
    const size_t rot = (size_t)n_groups * (n_members + 1) * L * ctx->c->n;
    return (rot + shm::shared_rotate_ws_words(*ctx->c, n_groups, n_members, L)) * 8;
}

// the reference's order (ShRotate.cu:218-256): the automorphism on a and every b first, then
// ModUp of the rotated a, the inner products and ModDown; the hoisted entry point with the
// identity element runs the key-switch half
int shm_shared_rotate(const shm_context *ctx, const uint64_t *sh, uint32_t n_groups, uint32_t n_members, uint32_t elt,
                      const uint64_t *key, uint64_t *out, uint32_t L, void *workspace, size_t workspace_bytes,
                      void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        if (!key || !out || n_members == 0) throw std::invalid_argument("bad shared-a rotation arguments");
        if (out == sh) throw std::invalid_argument("the output must not alias the input");
        if (elt % 2 == 0 || elt >= 2 * c.n) throw std::invalid_argument("Galois element must be odd and below 2N");
        set_device(c);
        const size_t rot = (size_t)n_groups * (n_members + 1) * L * c.n;
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, rot + shm::shared_rotate_ws_words(c, n_groups, n_members, L));
        shm::apply_galois(c, sh, ws, (uint32_t)((size_t)n_groups * (n_members + 1) * L), elt, S(stream));
        const uint32_t one = 1;
        const uint64_t *k = key;
        uint64_t *o = out;
        shm::shared_rotate_hoisted(c, ws, n_groups, n_members, L, 1, &one, &k, &o, ws + rot, S(stream));
    });
}

size_t shm_fmt_switch_forward_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                              uint32_t L) {
    return ctx && ctx->c ? shm::fmt_forward_ws_words(*ctx->c, n_groups, n_members, L) * 8 : 0;
}

int shm_fmt_switch_forward(const shm_context *ctx, const uint64_t *cts, uint32_t n_groups, uint32_t n_members,
                           const uint64_t *key, uint64_t *out, uint32_t L, void *workspace, size_t workspace_bytes,
                           void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        if (!key || n_members == 0) throw std::invalid_argument("bad format-switch arguments");
        set_device(c);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, shm::fmt_forward_ws_words(c, n_groups, n_members, L));
        shm::fmt_forward(c, cts, n_groups, n_members, L, key, out, ws, S(stream));
    });
}

size_t shm_fmt_switch_backward_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                               uint32_t L) {
    return ctx && ctx->c ? shm::fmt_backward_ws_words(*ctx->c, n_groups, n_members, L) * 8 : 0;
}

int shm_fmt_switch_backward(const shm_context *ctx, const uint64_t *sh, uint32_t n_groups, uint32_t n_members,
                            const uint64_t *const *keys, uint64_t *out, uint32_t L, void *workspace,
                            size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        if (!keys || n_members == 0) throw std::invalid_argument("bad format-switch arguments");
        set_device(c);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, shm::fmt_backward_ws_words(c, n_groups, n_members, L));
        shm::fmt_backward(c, sh, n_groups, n_members, L, keys, out, ws, S(stream));
    });
}

// ---- extended basis

static void check_ext(const shm::Context &c, uint32_t L) {
    if (c.np == 0) throw std::invalid_argument("context has no special primes");
    if (L < 1 || L > c.nq) throw std::invalid_argument("level out of range");
}

int shm_extend(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
               void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_ext(c, L);
        set_device(c);
        shm::extend(c, in, out, n_polys, L, S(stream));
    });
}

int shm_add_ext(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys,
                uint32_t L, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_ext(c, L);
        set_device(c);
        shm::add_ext(c, a, b, out, n_polys, L, S(stream));
    });
}

size_t shm_moddown_ext_workspace_bytes(const shm_context *ctx, uint32_t n_polys, uint32_t L) {
    return ctx && ctx->c ? shm::moddown_ext_ws_words(*ctx->c, n_polys, L) * 8 : 0;
}

int shm_moddown_ext(const shm_context *ctx, uint64_t *ext, uint64_t *out, uint32_t n_polys, uint32_t L,
                    void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_ext(c, L);
        set_device(c);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, shm::moddown_ext_ws_words(c, n_polys, L));
        shm::moddown_ext(c, ext, out, n_polys, L, ws, S(stream));
    });
}

int shm_multiply_plain_accumulate_ext(const shm_context *ctx, const uint64_t *const *X, const uint64_t *const *P,
                                      uint32_t k, uint64_t *out, uint32_t n_polys, uint32_t L, int accumulate,
                                      void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_ext(c, L);
        if (!X || !P) throw std::invalid_argument("null term arrays");
        set_device(c);
        // sum of `chunk` products must stay below the Barrett bound 2^(63 + bits(q)) of every limb
        uint32_t chunk = shm::kMaxAccTerms;
        for (uint32_t i = 0; i < L + c.np; i++) {
            const uint64_t q = c.primes[i < L ? i : c.nq + (i - L)];
            int b = shm::host::bit_length(q);
            uint32_t lim = 2 * b >= 63 + b ? 1u : (63 + b - 2 * b >= 5 ? 32u : (1u << (63 + b - 2 * b)));
            chunk = std::min(chunk, lim);
        }
        for (uint32_t t0 = 0; t0 < k; t0 += chunk) {
            uint32_t kk = std::min(chunk, k - t0);
            shm::PtrTab x{}, p{};
            for (uint32_t t = 0; t < kk; t++) {
                x.p[t] = X[t0 + t];
                p.p[t] = P[t0 + t];
            }
            shm::mul_plain_acc(c, x, p, kk, out, n_polys, L, accumulate || t0 > 0, S(stream), true);
        }
    });
}

int shm_lift_signed_ext(const shm_context *ctx, const int64_t *coeffs, uint64_t *out, uint32_t n_polys, uint32_t L,
                        void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_ext(c, L);
        set_device(c);
        shm::lift_signed_ext(c, coeffs, out, n_polys, L, S(stream));
    });
}

int shm_ntt_forward_ext(const shm_context *ctx, uint64_t *data, uint32_t n_polys, uint32_t L, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_ext(c, L);
        set_device(c);
        const uint32_t LP = L + c.np;
        shm::ntt_forward(c, data, n_polys * LP, LP, shm::ext_map(L, c), S(stream));
    });
}

size_t shm_shared_rotate_ext_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                             uint32_t L) {
    return ctx && ctx->c ? shm::shared_rotate_ext_ws_words(*ctx->c, n_groups, n_members, L) * 8 : 0;
}

int shm_shared_rotate_ext(const shm_context *ctx, const uint64_t *in, int in_ext, uint32_t n_groups,
                          uint32_t n_members, uint32_t n_elts, const uint32_t *elts, const uint64_t *const *keys,
                          uint64_t *const *outs, uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_ext(c, L);
        if (n_elts && (!elts || !keys || !outs)) throw std::invalid_argument("null element arrays");
        if (n_members == 0) throw std::invalid_argument("groups need at least one member");
        set_device(c);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, shm::shared_rotate_ext_ws_words(c, n_groups, n_members, L));
        shm::shared_rotate_ext(c, in, in_ext != 0, n_groups, n_members, L, n_elts, elts, keys, outs, ws, S(stream));
    });
}

int shm_rotate(const shm_context *ctx, const uint64_t *ct, int step, const uint64_t *galois_key, uint64_t *out,
               uint32_t n_cts, uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    uint32_t elt = shm_galois_elt_from_step(ctx, step);
    if (!elt) {
        g_err = "rotation step out of range";
        return SHM_EINVAL;
    }
    return shm_apply_galois(ctx, ct, elt, galois_key, out, n_cts, L, workspace, workspace_bytes, stream);
}

static shm::ScalarTab scalar_tab(const shm::Context &c, const uint64_t *scalars, uint32_t L) {
    if (!scalars) throw std::invalid_argument("null scalars");
    if (L > 64) throw std::invalid_argument("at most 64 limbs for scalar operations");
    shm::ScalarTab s{};
    for (uint32_t i = 0; i < L; i++) {
        uint64_t q = c.primes[i];
        if (scalars[i] >= q) throw std::invalid_argument("scalar residue must be below its prime");
        s.v[i] = scalars[i];
        s.shoup[i] = shm::host::shoup_of(scalars[i], q);
    }
    return s;
}

int shm_multiply_scalar(const shm_context *ctx, const uint64_t *a, const uint64_t *scalars, uint64_t *out,
                        uint32_t n_polys, uint32_t L, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        set_device(c);
        shm::mul_scalar(c, a, out, scalar_tab(c, scalars, L), n_polys, L, S(stream));
    });
}

int shm_add_scalar(const shm_context *ctx, const uint64_t *a, const uint64_t *scalars, uint64_t *out,
                   uint32_t n_cts, uint32_t L, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        set_device(c);
        shm::add_scalar(c, a, out, scalar_tab(c, scalars, L), n_cts, L, S(stream));
    });
}

int shm_linear_combination(const shm_context *ctx, const uint64_t *const *X, const uint32_t *X_levels,
                           const uint64_t *w, uint32_t k, const uint64_t *w0, uint64_t *out, uint32_t n_cts,
                           uint32_t L, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        if (!X || !X_levels || !w) throw std::invalid_argument("null term arrays");
        if (k < 1 || k > (uint32_t)shm::kMaxLinTerms) throw std::invalid_argument("linear combination of 1..8 terms");
        if (L > 64) throw std::invalid_argument("level out of range");
        set_device(c);
        std::unique_ptr<shm::LinTerms> t(new shm::LinTerms{});
        t->k = k;
        for (uint32_t i = 0; i < k; i++) {
            t->x[i] = X[i];
            t->levels[i] = X_levels[i];
            for (uint32_t l = 0; l < L; l++) {
                const uint64_t q = c.primes[l], v = w[(size_t)i * L + l];
                if (v >= q) throw std::invalid_argument("weights must be residues below their prime");
                t->w[i][l] = v;
                t->ws[i][l] = shm::host::shoup_of(v, q);
            }
        }
        t->has_w0 = w0 ? 1 : 0;
        for (uint32_t l = 0; w0 && l < L; l++) {
            if (w0[l] >= c.primes[l]) throw std::invalid_argument("constant residues must be below their prime");
            t->w0[l] = w0[l];
        }
        shm::linear_combination(c, *t, out, n_cts, L, S(stream));
    });
}

int shm_multiply_plain_accumulate(const shm_context *ctx, const uint64_t *const *X, const uint64_t *const *P,
                                  uint32_t k, uint64_t *out, uint32_t n_polys, uint32_t L, int accumulate,
                                  void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        if (!X || !P) throw std::invalid_argument("null term arrays");
        set_device(c);
        // sum of `chunk` products must stay below the Barrett bound 2^(63 + bits(q))
        uint32_t chunk = shm::kMaxAccTerms;
        for (uint32_t i = 0; i < L; i++) {
            int b = shm::host::bit_length(c.primes[i]);
            uint32_t lim = 2 * b >= 63 + b ? 1u : (63 + b - 2 * b >= 5 ? 32u : (1u << (63 + b - 2 * b)));
            chunk = std::min(chunk, lim);
        }
        for (uint32_t t0 = 0; t0 < k; t0 += chunk) {
            uint32_t kk = std::min(chunk, k - t0);
            shm::PtrTab x{}, p{};
            for (uint32_t t = 0; t < kk; t++) {
                x.p[t] = X[t0 + t];
                p.p[t] = P[t0 + t];
            }
            shm::mul_plain_acc(c, x, p, kk, out, n_polys, L, accumulate || t0 > 0, S(stream));
        }
    });
}

size_t shm_modraise_workspace_bytes(const shm_context *ctx, uint32_t n_polys) {
    return ctx && ctx->c ? (size_t)n_polys * ctx->c->n * 8 : 0;
}

int shm_modraise(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
                 void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        set_device(c);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, (size_t)n_polys * c.n);
        shm::modraise(c, in, out, n_polys, L, ws, S(stream));
    });
}

int shm_drop_limbs(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L_in,
                   uint32_t L_out, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L_in);
        if (L_out < 1 || L_out > L_in) throw std::invalid_argument("L_out must be in [1, L_in]");
        set_device(c);
        const size_t n = c.n;
        SHM_CUDA(cudaMemcpy2DAsync(out, L_out * n * 8, in, L_in * n * 8, L_out * n * 8, n_polys,
                                   cudaMemcpyDeviceToDevice, S(stream)));
    });
}

// ---- device memory of the host library

int shm_malloc(const shm_context *ctx, size_t bytes, void **out, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        if (!out) throw std::invalid_argument("null output pointer");
        *out = nullptr;
        set_device(c);
        cudaMemPool_t pool = c.mempool();
        if (bytes == 0) return;
        cudaError_t e = cudaMallocFromPoolAsync(out, bytes, pool, S(stream));
        if (e == cudaErrorMemoryAllocation) {
            // blocks freed on other streams become reusable once their work is done: wait for
            // the device once and retry before reporting out of memory
            cudaGetLastError();
            if (std::getenv("SHMOAI_POOL_TRACE"))
                std::fprintf(stderr, "shm_malloc: %.2f GB found no room: waiting for the device\n", bytes / 1e9);
            SHM_CUDA(cudaDeviceSynchronize());
            e = cudaMallocFromPoolAsync(out, bytes, pool, S(stream));
        }
        if (e == cudaErrorMemoryAllocation) {
            // the free blocks may be scattered over the pool's chunks with none large enough:
            // give every wholly free chunk back to the device and try once more
            cudaGetLastError();
            if (std::getenv("SHMOAI_POOL_TRACE")) {
                uint64_t reserved = 0, used = 0;
                cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
                cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
                std::fprintf(stderr, "shm_malloc: %.2f GB found no room (pool %.2f GB used, %.2f GB reserved): trimming\n",
                             bytes / 1e9, used / 1e9, reserved / 1e9);
            }
            SHM_CUDA(cudaMemPoolTrimTo(pool, 0));
            e = cudaMallocFromPoolAsync(out, bytes, pool, S(stream));
        }
        SHM_CUDA(e);
    });
}

int shm_pool_usage(const shm_context *ctx, size_t *reserved, size_t *used, size_t *used_high, int reset_high) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        set_device(c);
        cudaMemPool_t pool = c.mempool();
        uint64_t v = 0;
        if (reserved) {
            SHM_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &v));
            *reserved = v;
        }
        if (used) {
            SHM_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &v));
            *used = v;
        }
        if (used_high) {
            SHM_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &v));
            *used_high = v;
        }
        if (reset_high) {
            uint64_t zero = 0;
            SHM_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero));
        }
    });
}

int shm_free(const shm_context *ctx, void *ptr, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        if (!ptr) return;
        set_device(c);
        SHM_CUDA(cudaFreeAsync(ptr, S(stream)));
    });
}

int shm_memcpy(const shm_context *ctx, void *dst, const void *src, size_t bytes, int kind, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        cudaMemcpyKind k = kind == SHM_COPY_H2D   ? cudaMemcpyHostToDevice
                           : kind == SHM_COPY_D2H ? cudaMemcpyDeviceToHost
                           : kind == SHM_COPY_D2D ? cudaMemcpyDeviceToDevice
                                                  : throw std::invalid_argument("bad copy kind");
        if (!bytes) return;
        set_device(c);
        SHM_CUDA(cudaMemcpyAsync(dst, src, bytes, k, S(stream)));
        if (kind != SHM_COPY_D2D) SHM_CUDA(cudaStreamSynchronize(S(stream)));  // host buffers may be pageable
    });
}

int shm_synchronize(const shm_context *ctx, void *stream) {
    return guard([&] {
        set_device(ctx_of(ctx));
        SHM_CUDA(cudaStreamSynchronize(S(stream)));
    });
}

int shm_stream_create(const shm_context *ctx, void **stream) {
    return guard([&] {
        if (!stream) throw std::invalid_argument("null output pointer");
        set_device(ctx_of(ctx));
        cudaStream_t s = nullptr;
        SHM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        *stream = s;
    });
}

int shm_stream_destroy(const shm_context *ctx, void *stream) {
    return guard([&] {
        set_device(ctx_of(ctx));
        if (stream) SHM_CUDA(cudaStreamDestroy(S(stream)));
    });
}

// ---- CUDA graphs

struct shm_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;
    int device = 0;
};

int shm_graph_begin(const shm_context *ctx, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        if (!stream) throw std::invalid_argument("the legacy default stream cannot be captured");
        set_device(c);
        // blocks the pool keeps for reuse would sit beside the graph's own allocations
        SHM_CUDA(cudaStreamSynchronize(S(stream)));
        SHM_CUDA(cudaMemPoolTrimTo(c.mempool(), 0));
        SHM_CUDA(cudaStreamBeginCapture(S(stream), cudaStreamCaptureModeThreadLocal));
    });
}

int shm_graph_end(const shm_context *ctx, void *stream, shm_graph **out) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        if (!out) throw std::invalid_argument("null output pointer");
        *out = nullptr;
        set_device(c);
        std::unique_ptr<shm_graph> g(new shm_graph);
        g->device = c.device;
        SHM_CUDA(cudaStreamEndCapture(S(stream), &g->graph));
        size_t n = 0;
        SHM_CUDA(cudaGraphGetNodes(g->graph, nullptr, &n));
        std::vector<cudaGraphNode_t> nodes(n);
        if (n) SHM_CUDA(cudaGraphGetNodes(g->graph, nodes.data(), &n));
        for (cudaGraphNode_t nd : nodes) {
            cudaGraphNodeType t;
            SHM_CUDA(cudaGraphNodeGetType(nd, &t));
            if (t == cudaGraphNodeTypeKernel) g->kernels++;
        }
        // no auto-free: a replay fails loudly if the recorded calls left an allocation alive
        SHM_CUDA(cudaGraphInstantiateWithFlags(&g->exec, g->graph, 0));
        *out = g.release();
    });
}

int shm_graph_launch(const shm_graph *g, void *stream) {
    return guard([&] {
        if (!g || !g->exec) throw std::invalid_argument("null graph");
        SHM_CUDA(cudaSetDevice(g->device));
        SHM_CUDA(cudaGraphLaunch(g->exec, S(stream)));
        SHM_LAUNCHED(g->kernels);
    });
}

uint64_t shm_graph_kernels(const shm_graph *g) { return g ? g->kernels : 0; }

// ---- autotuning

int shm_autotune(shm_context *ctx, int knob, uint32_t size, uint32_t level, uint32_t members, float *times,
                 uint32_t cap, uint32_t *chosen) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        set_device(c);
        std::vector<float> ms;
        uint32_t best;
        if (knob == SHM_TUNE_NTT_TILE)
            best = shm::tune_ntt_tile(c, size, ms);
        else if (knob == SHM_TUNE_IP_CHUNK)
            best = shm::tune_ip_chunk(c, size, level, members, ms);
        else
            throw std::invalid_argument("unknown tuning knob");
        for (uint32_t i = 0; times && i < cap && i < ms.size(); i++) times[i] = ms[i];
        if (chosen) *chosen = best;
    });
}

int shm_tune_get(const shm_context *ctx, int knob, uint32_t *index) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        if (!index) throw std::invalid_argument("null output pointer");
        if (knob == SHM_TUNE_NTT_TILE) {
            *index = (uint32_t)c.ntt_variant;
        } else if (knob == SHM_TUNE_IP_CHUNK) {
            const uint32_t *b = std::begin(shm::kIpChunkCandidates), *e = std::end(shm::kIpChunkCandidates);
            *index = (uint32_t)(std::find(b, e, c.ip_chunk_bytes) - b);
        } else {
            throw std::invalid_argument("unknown tuning knob");
        }
    });
}

int shm_tune_set(shm_context *ctx, int knob, uint32_t index) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        set_device(c);
        if (knob == SHM_TUNE_NTT_TILE) {
            if (index >= (uint32_t)shm::kNttVariantCount) throw std::invalid_argument("tile variant out of range");
            SHM_CUDA(cudaDeviceSynchronize());  // launches in flight keep their shape
            c.ntt_variant = (int)index;
        } else if (knob == SHM_TUNE_IP_CHUNK) {
            if (index >= std::size(shm::kIpChunkCandidates)) throw std::invalid_argument("chunk candidate out of range");
            SHM_CUDA(cudaDeviceSynchronize());
            c.ip_chunk_bytes = shm::kIpChunkCandidates[index];
        } else {
            throw std::invalid_argument("unknown tuning knob");
        }
    });
}

void shm_graph_destroy(shm_graph *g) {
    if (!g) return;
    cudaSetDevice(g->device);
    if (g->exec) {
        cudaDeviceSynchronize();  // a replay may still run
        cudaGraphExecDestroy(g->exec);
    }
    if (g->graph) cudaGraphDestroy(g->graph);
    cudaDeviceGraphMemTrim(g->device);
    delete g;
    (void)cudaGetLastError();
}

// ---- sampling and lifting

int shm_sample_uniform(const shm_context *ctx, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t seed,
                       void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        set_device(c);
        shm::sample_uniform(c, out, n_polys, L, seed, S(stream));
    });
}

int shm_sample_cbd(const shm_context *ctx, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t seed,
                   void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        set_device(c);
        shm::sample_cbd(c, out, n_polys, L, seed, S(stream));
    });
}

size_t shm_encode_workspace_bytes(const shm_context *ctx, uint32_t n_vectors) {
    return ctx && ctx->c ? shm::encode_ws_bytes(*ctx->c, n_vectors) : 0;
}

int shm_encode(const shm_context *ctx, const double *re, const double *im, uint32_t n_vectors, uint32_t n_values,
               double scale, int64_t *coeffs, void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        if (n_values && (!re || !im)) throw std::invalid_argument("null slot arrays");
        set_device(c);
        void *ws = ws_of(c, workspace, workspace_bytes, (shm::encode_ws_bytes(c, n_vectors) + 7) / 8);
        if (!shm::encode(c, re, im, n_vectors, n_values, scale, coeffs, ws, S(stream)))
            throw std::invalid_argument("encoded values are too large");
    });
}

int shm_decode(const shm_context *ctx, const double *coeffs, uint32_t n_vectors, double scale, double *re, double *im,
               void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        set_device(c);
        void *ws = ws_of(c, workspace, workspace_bytes, (shm::encode_ws_bytes(c, n_vectors) + 7) / 8);
        shm::decode(c, coeffs, n_vectors, scale, re, im, ws, S(stream));
    });
}

int shm_lift_signed(const shm_context *ctx, const int64_t *coeffs, uint64_t *out, uint32_t n_polys, uint32_t L,
                    void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        set_device(c);
        shm::lift_signed(c, coeffs, out, n_polys, L, S(stream));
    });
}

size_t shm_ctpt_matmul_workspace_bytes(const shm_context *ctx, uint32_t n_in, uint32_t n_out, uint32_t L) {
    return ctx && ctx->c ? shm::ctpt_ws_words(*ctx->c, n_in, n_out, L) * 8 : 0;
}

int shm_ctpt_matmul(const shm_context *ctx, const uint64_t *X, const int64_t *W, uint64_t *Y, uint32_t n_in,
                    uint32_t n_out, uint32_t L, void *workspace, size_t workspace_bytes, void *stream) {
    return guard([&] {
        auto &c = const_cast<shm::Context &>(ctx_of(ctx));
        check_level(c, L);
        set_device(c);
        uint64_t *ws = ws_of(c, workspace, workspace_bytes, shm::ctpt_ws_words(c, n_in, n_out, L));
        shm::ctpt_matmul(c, X, W, Y, n_in, n_out, L, ws, S(stream));
    });
}

int shm_ctpt_matmul_cuda_core(const shm_context *ctx, const uint64_t *X, const int64_t *W, uint64_t *Y,
                              uint32_t n_in, uint32_t n_out, uint32_t L, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        set_device(c);
        shm::ctpt_matmul_cuda_core(c, X, W, Y, n_in, n_out, L, S(stream));
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Rescale for callers that cannot allocate device memory.
//
// Some hosts own every byte of device memory through their own pool and forbid
// direct cudaMalloc (a serving runtime with a fixed memory budget), some cannot
// afford cudaMalloc's implicit device-wide synchronisation on a latency-critical
// path, and some FFI callers have no device allocator binding at all.  For them
// shm_rescale_noalloc runs the same rescale as shm_rescale but takes its scratch
// from the fixed array below instead of a caller workspace or the context arena.

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB, held by every GPU that loads the library
static __device__ __align__(256) uint64_t g_noalloc_scratch[kNoAllocScratchBytes / 8];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
uint64_t *g_noalloc_addr[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current).  The
// host-side symbol g_noalloc_scratch is only a stand-in and must never be passed
// to a kernel; the address comes from cudaGetSymbolAddress, once per device.
uint64_t *noalloc_scratch(int device) {
    if (device < 0 || device >= kMaxDevices) throw std::invalid_argument("device index out of range");
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void *p = nullptr;
        SHM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_addr[device] = static_cast<uint64_t *>(p);
    }
    return g_noalloc_addr[device];
}

}  // namespace

extern "C" size_t shm_rescale_noalloc_max_words(void) { return kNoAllocScratchBytes / 8; }

extern "C" int shm_rescale_noalloc(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys,
                                   uint32_t L, void *stream) {
    return guard([&] {
        auto &c = ctx_of(ctx);
        check_level(c, L);
        if (L < 2 || L > c.nq) throw std::invalid_argument("rescale needs 2 <= L <= n_q limbs");
        const size_t need = shm::rescale_ws_words(c, n_polys, L);
        if (need > kNoAllocScratchBytes / 8)
            throw std::invalid_argument("shm_rescale_noalloc: n_polys * L * N exceeds the fixed scratch of " +
                                        std::to_string(kNoAllocScratchBytes / 8) + " words (32 MiB)");
        set_device(c);
        shm::rescale(c, in, out, n_polys, L, noalloc_scratch(c.device), S(stream));
    });
}
