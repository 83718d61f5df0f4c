// extern "C" entry points of include/shmoai_host.h over the C++ host classes.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>

#include "../../include/shmoai_host.h"
#include "../../include/shmoai/wire.hpp"
#include "internal.hpp"

using namespace shmoai;

struct shm_host {
    std::unique_ptr<Context> ctx;
    std::unique_ptr<Encoder> enc;
    std::unique_ptr<KeyGenerator> kg;
    std::unique_ptr<Evaluator> ev;
    DeviceBuffer relin;
    std::unique_ptr<PublicEncryptor> pub;  // shm_host_gen_public_key
    std::map<uint32_t, DeviceBuffer> galois;
    std::map<uint32_t, SharedAKeys> shared;  // group size -> keys

    void use_shared(uint32_t members) {
        auto it = shared.find(members);
        if (it == shared.end()) throw Error("no shared-a keys for groups of " + std::to_string(members));
        ev->shared_keys = &it->second;
    }
};

struct shm_ct {
    Ciphertext ct;
};

struct shm_boot {
    shm_host *h;
    std::unique_ptr<BatchBootstrapper> b;
};

struct shm_host_graph {
    std::unique_ptr<Graph> g;
};

struct shm_server {
    std::unique_ptr<Server> s;
};

namespace {

thread_local std::string g_err;

template <typename F>
int guard(F &&f) {
    try {
        f();
        return SHM_OK;
    } catch (const Error &e) {
        g_err = e.what();
        return e.code;
    } catch (const std::bad_alloc &) {
        g_err = "host out of memory";
        return SHM_ENOMEM;
    } catch (const std::exception &e) {
        g_err = e.what();
        return SHM_EINTERNAL;
    } catch (...) {
        g_err = "unknown error";
        return SHM_EINTERNAL;
    }
}

shm_host &H(shm_host *h) {
    if (!h || !h->ctx) throw Error("null host handle");
    return *h;
}

const Ciphertext &C(const shm_ct *c) {
    if (!c) throw Error("null ciphertext handle");
    return c->ct;
}

void put(shm_ct **out, Ciphertext &&ct) {
    if (!out) throw Error("null output handle");
    *out = new shm_ct{std::move(ct)};
}

void prepare_for(shm_host &h, const Ciphertext &a) {
    if (a.shared) h.use_shared(a.members());
}

void finish_create(shm_host *h, uint32_t hw, uint64_t seed) {
    h->enc.reset(new Encoder(*h->ctx));
    h->kg.reset(new KeyGenerator(*h->ctx, hw, seed));
    h->ev.reset(new Evaluator(*h->ctx, *h->enc));
    h->ev->relin_key = &h->relin;
    h->ev->galois_keys = &h->galois;
}

}  // namespace

extern "C" {

const char *shm_host_last_error(void) { return g_err.c_str(); }

int shm_host_create(shm_host **out, uint32_t log_n, const uint64_t *primes, uint32_t n_primes, uint32_t n_special,
                    int device, uint32_t hamming_weight, uint64_t seed) {
    return guard([&] {
        if (!out || !primes) throw Error("null argument");
        std::unique_ptr<shm_host> h(new shm_host);
        h->ctx.reset(new Context(log_n, std::vector<uint64_t>(primes, primes + n_primes), n_special, device));
        finish_create(h.get(), hamming_weight, seed);
        *out = h.release();
    });
}

int shm_host_create_from_bits(shm_host **out, uint32_t log_n, const int *bits, uint32_t n_primes,
                              uint32_t n_special, int device, uint32_t hamming_weight, uint64_t seed) {
    return guard([&] {
        if (!out || !bits) throw Error("null argument");
        std::unique_ptr<shm_host> h(new shm_host);
        h->ctx.reset(new Context(log_n, std::vector<int>(bits, bits + n_primes), n_special, device));
        finish_create(h.get(), hamming_weight, seed);
        *out = h.release();
    });
}

void shm_host_destroy(shm_host *h) {
    if (!h) return;
    // keys and buffers are returned to the context's pool before the context goes
    h->ev.reset();
    h->pub.reset();
    h->kg.reset();
    h->shared.clear();
    h->galois.clear();
    h->relin = DeviceBuffer();
    h->enc.reset();
    h->ctx.reset();
    delete h;
}

const shm_context *shm_host_context(const shm_host *h) { return h && h->ctx ? h->ctx->handle() : nullptr; }

int shm_host_primes(const shm_host *h, uint64_t *out) {
    return guard([&] {
        if (!h || !h->ctx || !out) throw Error("null argument");
        std::copy(h->ctx->primes.begin(), h->ctx->primes.end(), out);
    });
}

int shm_host_synchronize(shm_host *h) {
    return guard([&] { H(h).ctx->synchronize(); });
}

int shm_host_device_memory(shm_host *h, size_t *in_use, size_t *peak, int reset_peak) {
    return guard([&] {
        auto &hh = H(h);
        hh.ctx->check(shm_pool_usage(hh.ctx->handle(), nullptr, in_use, peak, reset_peak));
    });
}

int shm_host_gen_relin_key(shm_host *h) {
    return guard([&] { H(h).relin = H(h).kg->relin_key(); });
}

int shm_host_gen_galois_keys(shm_host *h, const uint32_t *elts, uint32_t n_elts) {
    return guard([&] {
        auto &hh = H(h);
        for (uint32_t i = 0; i < n_elts; i++)
            if (!hh.galois.count(elts[i])) hh.galois.emplace(elts[i], hh.kg->galois_key(elts[i]));
    });
}

int shm_host_gen_shared_keys(shm_host *h, uint32_t members, uint32_t hamming_weight, const uint32_t *elts,
                             uint32_t n_elts) {
    return guard([&] {
        auto &hh = H(h);
        if (!members) throw Error("group size must be positive");
        hh.ev->shared_keys = nullptr;
        hh.shared.erase(members);
        hh.shared.emplace(members, hh.kg->shared_keys(members, std::vector<uint32_t>(elts, elts + n_elts),
                                                      hamming_weight));
    });
}

uint32_t shm_host_galois_elt(const shm_host *h, int step) {
    return h && h->ev ? h->ev->galois_elt(step) : 0;
}

int shm_host_encrypt(shm_host *h, const double *re, const double *im, uint32_t count, uint32_t n_values, uint32_t L,
                     double scale, shm_ct **out) {
    return guard([&] {
        auto &hh = H(h);
        std::vector<std::vector<cplx>> z(count, std::vector<cplx>(n_values));
        for (uint32_t i = 0; i < count; i++)
            for (uint32_t j = 0; j < n_values; j++)
                z[i][j] = cplx(re[(size_t)i * n_values + j], im ? im[(size_t)i * n_values + j] : 0.0);
        put(out, hh.kg->encrypt(z, scale, L));
    });
}

int shm_host_gen_public_key(shm_host *h, uint64_t seed) {
    return guard([&] {
        auto &hh = H(h);
        hh.pub = std::make_unique<PublicEncryptor>(*hh.ctx, hh.kg->public_key(), seed);
    });
}

int shm_host_encrypt_public(shm_host *h, const double *re, const double *im, uint32_t count, uint32_t n_values,
                            uint32_t L, double scale, shm_ct **out) {
    return guard([&] {
        auto &hh = H(h);
        if (!hh.pub) throw Error("no public key: call shm_host_gen_public_key first");
        std::vector<std::vector<cplx>> z(count, std::vector<cplx>(n_values));
        for (uint32_t i = 0; i < count; i++)
            for (uint32_t j = 0; j < n_values; j++)
                z[i][j] = cplx(re[(size_t)i * n_values + j], im ? im[(size_t)i * n_values + j] : 0.0);
        put(out, hh.pub->encrypt(z, scale, L));
    });
}

int shm_host_batch_input(shm_host *h, const double *X, uint32_t num_X, uint32_t num_row, uint32_t num_col,
                         double scale, uint32_t L, shm_ct **out) {
    return guard([&] {
        auto &hh = H(h);
        if (!hh.pub) throw Error("no public key: call shm_host_gen_public_key first");
        std::vector<double> x(X, X + (size_t)num_X * num_row * num_col);
        put(out, batch_input(*hh.pub, x, num_X, num_row, num_col, scale, L));
    });
}

int shm_host_bias_vec(const int *lengths, uint32_t num_X, uint32_t num_row, int *out) {
    return guard([&] {
        std::vector<int> v = bias_vec(std::vector<int>(lengths, lengths + num_X), num_X, num_row);
        std::copy(v.begin(), v.end(), out);
    });
}

int shm_host_decrypt(shm_host *h, const shm_ct *ct, double *re, double *im) {
    return guard([&] {
        auto &hh = H(h);
        // shared-a groups decrypt with the auxiliary secrets of the last shm_host_gen_shared_keys
        std::vector<std::vector<cplx>> z = hh.kg->decrypt(C(ct));
        const size_t slots = hh.ctx->n / 2;
        for (size_t r = 0; r < z.size(); r++)
            for (size_t j = 0; j < slots; j++) {
                re[r * slots + j] = z[r][j].real();
                if (im) im[r * slots + j] = z[r][j].imag();
            }
    });
}

int shm_ct_from_host(shm_host *h, const uint64_t *data, uint32_t count, uint32_t size, uint32_t L, double scale,
                     int shared, shm_ct **out) {
    return guard([&] {
        auto &hh = H(h);
        if (!count || !size || !L) throw Error("empty ciphertext batch");
        Ciphertext c;
        const size_t words = (size_t)count * size * L * hh.ctx->n;
        c.data = DeviceBuffer(*hh.ctx, words);
        c.count = count;
        c.size = size;
        c.L = L;
        c.scale_ = scale;
        c.shared = shared != 0;
        hh.ctx->check(shm_memcpy(hh.ctx->handle(), c.data.data(), data, words * 8, SHM_COPY_H2D, hh.ctx->stream()));
        put(out, std::move(c));
    });
}

int shm_ct_to_host(shm_host *h, const shm_ct *ct, uint64_t *data) {
    return guard([&] {
        auto &hh = H(h);
        const Ciphertext &c = C(ct);
        hh.ctx->check(shm_memcpy(hh.ctx->handle(), data, c.data.data(), c.polys() * c.L * hh.ctx->n * 8,
                                 SHM_COPY_D2H, hh.ctx->stream()));
    });
}

int shm_host_chebyshev(shm_host *h, const shm_ct *a, const double *coeffs, uint32_t n_coeffs, double lo, double hi,
                       shm_ct **out) {
    return guard([&] {
        auto &hh = H(h);
        if (!coeffs) throw Error("null coefficients");
        put(out, evaluate_chebyshev(*hh.ev, C(a), std::vector<double>(coeffs, coeffs + n_coeffs), lo, hi));
    });
}

int shm_host_gelu(shm_host *h, const shm_ct *a, shm_ct **out) {
    return guard([&] { put(out, gelu(*H(h).ev, C(a))); });
}

int shm_host_exp(shm_host *h, const shm_ct *a, shm_ct **out) {
    return guard([&] { put(out, exp_approx(*H(h).ev, C(a))); });
}

int shm_host_inverse(shm_host *h, const shm_ct *a, uint32_t iter, shm_ct **out) {
    return guard([&] { put(out, inverse_approx(*H(h).ev, C(a), (int)iter)); });
}

int shm_host_inv_sqrt(shm_host *h, const shm_ct *a, uint32_t d_newt, uint32_t d_gold, shm_ct **out) {
    return guard([&] { put(out, inv_sqrt_approx(*H(h).ev, C(a), (int)d_newt, (int)d_gold)); });
}

int shm_host_layernorm(shm_host *h, const shm_ct *a, const double *gamma, const double *beta, uint32_t d_newt,
                       uint32_t d_gold, shm_ct **out) {
    return guard([&] {
        auto &hh = H(h);
        const Ciphertext &x = C(a);
        if (!gamma || !beta) throw Error("null gamma or beta");
        put(out, layernorm(*hh.ev, x, std::vector<double>(gamma, gamma + x.count),
                           std::vector<double>(beta, beta + x.count), (int)d_newt, (int)d_gold));
    });
}

int shm_host_softmax(shm_host *h, const shm_ct *a, double shift, double sum_scale, uint32_t iter, shm_ct **out) {
    return guard([&] { put(out, softmax_batch(*H(h).ev, C(a), shift, sum_scale, (int)iter)); });
}

int shm_host_ct_ct_matmul(shm_host *h, const shm_ct *X, const shm_ct *W, uint32_t rows, uint32_t num_batch,
                          shm_ct **out) {
    return guard([&] { put(out, ct_ct_matmul_colpacking(*H(h).ev, C(X), C(W), rows, num_batch)); });
}

int shm_host_ct_ct_matmul_diag(shm_host *h, const shm_ct *X, const shm_ct *W, uint32_t num_batch, shm_ct **out) {
    return guard([&] { put(out, ct_ct_matmul_diagpacking(*H(h).ev, C(X), C(W), num_batch)); });
}

int shm_host_softmax_attention(shm_host *h, const shm_ct *a, const int *bias_vec, int input_num, uint32_t iter,
                               shm_ct **out) {
    return guard([&] {
        auto &hh = H(h);
        if (!bias_vec) throw Error("null bias_vec");
        put(out, softmax_attention(*hh.ev, C(a), std::vector<int>(bias_vec, bias_vec + hh.ctx->n / 2), input_num,
                                   (int)iter));
    });
}

int shm_host_chebyshev_capture(shm_host *h, const shm_ct *in, const double *coeffs, uint32_t n_coeffs, double lo,
                               double hi, shm_ct **out, shm_host_graph **graph) {
    return guard([&] {
        auto &hh = H(h);
        if (!graph || !out) throw Error("null output handle");
        std::vector<double> c = coeffs ? std::vector<double>(coeffs, coeffs + n_coeffs) : gelu_series();
        if (!coeffs) {
            lo = -19.5;
            hi = 12.5;
        }
        Ciphertext o;
        std::unique_ptr<Graph> g = capture_chebyshev(*hh.ev, C(in), c, lo, hi, o);
        *graph = new shm_host_graph{std::move(g)};
        put(out, std::move(o));
    });
}

int shm_ct_serialized_bytes(shm_host *h, const shm_ct *ct, size_t *bytes) {
    return guard([&] {
        if (!bytes) throw Error("null argument");
        *bytes = wire::serialized_bytes(*H(h).ctx, C(ct));
    });
}

int shm_ct_serialize(shm_host *h, const shm_ct *ct, void *buf, size_t cap) {
    return guard([&] {
        auto &hh = H(h);
        const size_t need = wire::serialized_bytes(*hh.ctx, C(ct));
        if (!buf || cap < need) throw Error("buffer smaller than the record (" + std::to_string(need) + " bytes)");
        uint8_t *p = static_cast<uint8_t *>(buf);
        size_t used = 0;
        wire::save([&](const void *src, size_t n) {
            if (used + n > need) throw Error("record larger than its computed size", SHM_EINTERNAL);
            std::memcpy(p + used, src, n);
            used += n;
        }, *hh.ctx, C(ct));
    });
}

int shm_ct_deserialize(shm_host *h, const void *buf, size_t len, shm_ct **out) {
    return guard([&] {
        auto &hh = H(h);
        if (!buf) throw Error("null argument");
        const uint8_t *p = static_cast<const uint8_t *>(buf);
        size_t used = 0;
        Ciphertext ct = wire::load_ciphertext([&](void *dst, size_t n) {
            if (n > len - used) throw Error("record truncated");
            std::memcpy(dst, p + used, n);
            used += n;
        }, *hh.ctx);
        if (used != len) throw Error("bytes after the record");
        put(out, std::move(ct));
    });
}

int shm_host_save_keys(shm_host *h, const char *path, int with_secrets) {
    return guard([&] {
        auto &hh = H(h);
        if (!path) throw Error("null path");
        std::ofstream f(path, std::ios::binary | std::ios::trunc);
        if (!f) throw Error(std::string("cannot open ") + path);
        wire::KeySet ks;
        if (with_secrets) {
            ks.secret = &hh.kg->secret_coeffs();
            ks.aux = &hh.kg->aux_secret_coeffs();
        }
        ks.relin = &hh.relin;
        ks.galois = &hh.galois;
        ks.shared = &hh.shared;
        wire::save_keys([&](const void *src, size_t n) {
            f.write(static_cast<const char *>(src), (std::streamsize)n);
            if (!f) throw Error(std::string("write failed: ") + path);
        }, *hh.ctx, ks);
        f.close();
        if (!f) throw Error(std::string("write failed: ") + path);
    });
}

int shm_host_load_keys(shm_host *h, const char *path) {
    return guard([&] {
        auto &hh = H(h);
        if (!path) throw Error("null path");
        std::ifstream f(path, std::ios::binary);
        if (!f) throw Error(std::string("cannot open ") + path);
        wire::LoadedKeys k = wire::load_keys([&](void *dst, size_t n) {
            f.read(static_cast<char *>(dst), (std::streamsize)n);
            if ((size_t)f.gcount() != n) throw Error("record truncated");
        }, *hh.ctx);
        if (f.peek() != std::char_traits<char>::eof()) throw Error("bytes after the end record");
        // everything was read and checked: install it
        if (k.has_secret) hh.kg->import_secrets(k.secret, k.aux);
        if (k.relin.data()) hh.relin = std::move(k.relin);
        for (auto &kv : k.galois) hh.galois[kv.first] = std::move(kv.second);
        hh.ev->shared_keys = nullptr;
        for (auto &kv : k.shared) {
            hh.shared.erase(kv.first);
            hh.shared.emplace(kv.first, std::move(kv.second));
        }
    });
}

int shm_host_import_secret_text(shm_host *h, const char *path) {
    return guard([&] {
        auto &hh = H(h);
        if (!path) throw Error("null path");
        std::ifstream f(path);
        if (!f) throw Error(std::string("cannot open ") + path);
        hh.kg->import_secrets(wire::import_secret_text(f, *hh.ctx), {});
    });
}

int shm_host_export_secret_text(shm_host *h, const char *path) {
    return guard([&] {
        auto &hh = H(h);
        if (!path) throw Error("null path");
        std::ofstream f(path, std::ios::trunc);
        if (!f) throw Error(std::string("cannot open ") + path);
        wire::export_secret_text(f, *hh.ctx, hh.kg->secret_coeffs());
        f.close();
        if (!f) throw Error(std::string("write failed: ") + path);
    });
}

int shm_host_import_key(shm_host *h, int kind, uint32_t elt, const uint64_t *words, size_t n_words) {
    return guard([&] {
        auto &hh = H(h);
        const Context &c = *hh.ctx;
        if (!words) throw Error("null argument");
        if (kind != SHM_KEY_RELIN && kind != SHM_KEY_GALOIS) throw Error("unknown key kind");
        const size_t QP = c.nq + c.np, want = (size_t)c.dnum * 2 * QP * c.n;
        if (n_words != want) throw Error("key of " + std::to_string(n_words) + " words, expected " + std::to_string(want));
        if (kind == SHM_KEY_GALOIS && (elt % 2 == 0 || elt >= 2 * c.n)) throw Error("invalid Galois element");
        for (size_t r = 0; r < (size_t)c.dnum * 2 * QP; r++) {
            const uint64_t q = c.primes[r % QP], *w = words + r * c.n;
            for (size_t k = 0; k < c.n; k++)
                if (w[k] >= q) throw Error("key residue not below its prime");
        }
        DeviceBuffer key(c, want);
        c.check(shm_memcpy(c.handle(), key.data(), words, want * 8, SHM_COPY_H2D, c.stream()));
        if (kind == SHM_KEY_RELIN) hh.relin = std::move(key);
        else hh.galois[elt] = std::move(key);
    });
}

int shm_ct_info(const shm_ct *ct, uint32_t *count, uint32_t *size, uint32_t *L, double *scale, int *shared) {
    return guard([&] {
        const Ciphertext &c = C(ct);
        if (count) *count = c.count;
        if (size) *size = c.size;
        if (L) *L = c.L;
        if (scale) *scale = c.scale_;
        if (shared) *shared = c.shared ? 1 : 0;
    });
}

int shm_host_encode(shm_host *h, const double *re, const double *im, uint32_t n_values, double scale,
                    int64_t *coeffs, int on_host) {
    return guard([&] {
        auto &hh = H(h);
        std::vector<cplx> z(n_values);
        for (uint32_t j = 0; j < n_values; j++) z[j] = cplx(re[j], im[j]);
        Encoder enc(*hh.ctx);
        std::vector<int64_t> c;
        if (on_host) {
            std::vector<double> f = enc.encode_float(z.data(), z.size(), scale);
            c.resize(f.size());
            for (size_t k = 0; k < f.size(); k++) {
                const double r = std::nearbyint(f[k]);
                if (!(std::fabs(r) < 4611686018427387904.0)) throw Error("encoded values are too large");
                c[k] = (int64_t)r;
            }
        } else {
            c = enc.encode_coeffs(z.data(), z.size(), scale);
        }
        std::copy(c.begin(), c.end(), coeffs);
    });
}

int shm_ct_write(shm_host *h, shm_ct *ct, const uint64_t *data) {
    return guard([&] {
        auto &hh = H(h);
        if (!ct) throw Error("null ciphertext handle");
        Ciphertext &c = ct->ct;
        hh.ctx->check(shm_memcpy(hh.ctx->handle(), c.data.data(), data, c.polys() * c.L * hh.ctx->n * 8,
                                 SHM_COPY_H2D, hh.ctx->stream()));
    });
}

const uint64_t *shm_ct_device_data(const shm_ct *ct) { return ct ? ct->ct.data.data() : nullptr; }

void shm_ct_destroy(shm_ct *ct) { delete ct; }

int shm_host_add(shm_host *h, const shm_ct *a, const shm_ct *b, shm_ct **out) {
    return guard([&] { put(out, H(h).ev->add(C(a), C(b))); });
}

int shm_host_sub(shm_host *h, const shm_ct *a, const shm_ct *b, shm_ct **out) {
    return guard([&] { put(out, H(h).ev->sub(C(a), C(b))); });
}

int shm_host_multiply(shm_host *h, const shm_ct *a, const shm_ct *b, shm_ct **out) {
    return guard([&] { put(out, H(h).ev->multiply(C(a), C(b), true)); });
}

int shm_host_rescale(shm_host *h, const shm_ct *a, shm_ct **out) {
    return guard([&] { put(out, H(h).ev->rescale_to_next(C(a))); });
}

int shm_host_multiply_const(shm_host *h, const shm_ct *a, double value, shm_ct **out) {
    return guard([&] { put(out, H(h).ev->multiply_const(C(a), value)); });
}

int shm_host_rotate(shm_host *h, const shm_ct *a, int step, shm_ct **out) {
    return guard([&] {
        prepare_for(H(h), C(a));
        put(out, H(h).ev->rotate_vector(C(a), step));
    });
}

int shm_host_conjugate(shm_host *h, const shm_ct *a, shm_ct **out) {
    return guard([&] {
        prepare_for(H(h), C(a));
        put(out, H(h).ev->complex_conjugate(C(a)));
    });
}

int shm_host_multiply_i(shm_host *h, const shm_ct *a, int sign, shm_ct **out) {
    return guard([&] { put(out, H(h).ev->multiply_i(C(a), sign)); });
}

int shm_host_slice(shm_host *h, const shm_ct *ct, uint32_t first, uint32_t count, shm_ct **out) {
    return guard([&] { put(out, H(h).ev->slice(C(ct), first, count)); });
}

int shm_host_ctpt_matmul(shm_host *h, const shm_ct *X, const int64_t *W, uint32_t n_out, double w_scale,
                         int tensor_cores, shm_ct **out) {
    return guard([&] {
        const Ciphertext &x = C(X);
        if (!W) throw Error("null weights");
        put(out, H(h).ev->ctpt_matmul(x, std::vector<int64_t>(W, W + (size_t)x.count * n_out), n_out, w_scale,
                                      tensor_cores != 0));
    });
}

int shm_host_ctpt_matmul_masked(shm_host *h, const shm_ct *X, const int64_t *W, uint32_t n_out, double w_scale,
                                const double *mask, int tensor_cores, shm_ct **out) {
    return guard([&] {
        const Ciphertext &x = C(X);
        if (!W || !mask) throw Error("null weights or mask");
        put(out, H(h).ev->ctpt_matmul_masked(x, std::vector<int64_t>(W, W + (size_t)x.count * n_out), n_out, w_scale,
                                             std::vector<double>(mask, mask + H(h).ctx->n / 2), tensor_cores != 0));
    });
}

int shm_host_to_shared(shm_host *h, const shm_ct *a, uint32_t members, shm_ct **out) {
    return guard([&] {
        H(h).use_shared(members);
        put(out, H(h).ev->to_shared(C(a), members));
    });
}

int shm_host_from_shared(shm_host *h, const shm_ct *a, shm_ct **out) {
    return guard([&] {
        prepare_for(H(h), C(a));
        put(out, H(h).ev->from_shared(C(a)));
    });
}

int shm_boot_create(shm_host *h, double scale, uint32_t input_level, shm_boot **out) {
    return guard([&] {
        auto &hh = H(h);
        if (!out) throw Error("null output handle");
        BootstrapParams p;
        p.scale = scale;
        p.input_level = input_level;
        std::unique_ptr<shm_boot> b(new shm_boot{h, std::unique_ptr<BatchBootstrapper>(new BatchBootstrapper(*hh.ev, p))});
        b->b->prepare();
        *out = b.release();
    });
}

void shm_boot_destroy(shm_boot *b) { delete b; }

int shm_boot_galois_elts(const shm_boot *b, uint32_t *out, uint32_t cap, uint32_t *n_out) {
    return guard([&] {
        if (!b) throw Error("null bootstrapper");
        std::vector<uint32_t> e = b->b->galois_elts();
        if (n_out) *n_out = (uint32_t)e.size();
        for (size_t i = 0; i < e.size() && i < cap; i++) out[i] = e[i];
    });
}

int shm_boot_run(shm_boot *b, const shm_ct *in, uint32_t members, shm_ct **out) {
    return guard([&] {
        if (!b) throw Error("null bootstrapper");
        if (members) {
            b->h->use_shared(members);
            put(out, b->b->bootstrap_shared_a_s2c_first(C(in), members));
        } else {
            put(out, b->b->bootstrap_ordinary_s2c_first(C(in)));
        }
    });
}

int shm_boot_run_c2s_first(shm_boot *b, const shm_ct *in, shm_ct **out) {
    return guard([&] {
        if (!b) throw Error("null bootstrapper");
        put(out, b->b->bootstrap_c2s_first(C(in)));
    });
}

int shm_boot_bert_layer(shm_boot *b, const shm_ct *X, const uint32_t *dims, const double *reals, const double *weights,
                        const int *bias_vec, shm_ct **out, double *stage_seconds) {
    return guard([&] {
        if (!b || !dims || !reals || !weights || !bias_vec) throw Error("null argument");
        BertLayerConfig cfg;
        cfg.hidden = dims[0];
        cfg.heads = dims[1];
        cfg.ffn = dims[2];
        cfg.num_X = dims[3];
        cfg.tokens = dims[4];
        cfg.input_num = dims[5];
        cfg.softmax_iter = (int)dims[6];
        cfg.ln_newt = (int)dims[7];
        cfg.ln_gold = (int)dims[8];
        cfg.gelu_input_level = dims[9];
        cfg.ffn_chunk = dims[10];
        cfg.members = dims[11];
        cfg.boot_batch = dims[12];
        cfg.w_scale = reals[0];
        cfg.ln_var_scale = reals[1];
        const size_t d = cfg.hidden, F = cfg.ffn;
        const double *p = weights;
        auto take = [&](size_t n) {
            std::vector<double> v(p, p + n);
            p += n;
            return v;
        };
        BertLayerWeights w;
        w.Wq = take(d * d);
        w.bq = take(d);
        w.Wk = take(d * d);
        w.bk = take(d);
        w.Wv = take(d * d);
        w.bv = take(d);
        w.Wo = take(d * d);
        w.bo = take(d);
        w.ln1_gamma = take(d);
        w.ln1_beta = take(d);
        w.Wi = take(d * F);
        w.bi = take(F);
        w.Wf = take(F * d);
        w.bf = take(d);
        w.ln2_gamma = take(d);
        w.ln2_beta = take(d);
        if (cfg.members) b->h->use_shared(cfg.members);
        Evaluator &ev = *b->h->ev;
        ev.galois_keys = &b->h->galois;
        std::vector<StageTime> t;
        const size_t slots = b->h->ctx->n / 2;
        // the attention's rotation keys: the host's own where it has them all, else made for the
        // attention block and released after it
        bool have_all = true;
        for (int st : bert_layer_rotation_steps(cfg, (uint32_t)slots))
            if (!b->h->galois.count(ev.galois_elt(st))) have_all = false;
        put(out, bert_layer(ev, *b->b, C(X), w, cfg, std::vector<int>(bias_vec, bias_vec + slots), &t,
                            have_all ? nullptr : b->h->kg.get()));
        if (stage_seconds)
            for (size_t i = 0; i < t.size(); i++) {
                stage_seconds[i] = t[i].seconds;
                stage_seconds[t.size() + i] = (double)t[i].peak_bytes / (double)(1ull << 30);
            }
    });
}

namespace {

std::string json_str(const std::string &v) {
    std::string o = "\"";
    for (char ch : v) {
        if (ch == '"' || ch == '\\') o += '\\';
        o += ch;
    }
    return o + "\"";
}

std::string tune_json(const std::vector<TuneRecord> &rs) {
    std::string o = "[";
    for (size_t i = 0; i < rs.size(); i++) {
        const TuneRecord &r = rs[i];
        o += (i ? ", " : "") + std::string("{\"knob\": ") + json_str(r.knob) + ", \"candidates\": [";
        for (size_t j = 0; j < r.candidates.size(); j++) o += (j ? ", " : "") + json_str(r.candidates[j]);
        o += "], \"ms\": [";
        for (size_t j = 0; j < r.ms.size(); j++) {
            char buf[64];
            snprintf(buf, sizeof buf, "%s%.6g", j ? ", " : "", r.ms[j]);
            o += buf;
        }
        o += "], \"chosen\": " + std::to_string(r.chosen) + "}";
    }
    return o + "]";
}

}  // namespace

int shm_boot_tune(shm_boot *b, uint32_t count, uint32_t members, char *json, size_t cap, size_t *needed) {
    return guard([&] {
        if (!b) throw Error("null bootstrapper");
        const std::string j = tune_json(b->b->tune(count, members));
        if (needed) *needed = j.size() + 1;
        if (json && cap) {
            const size_t n = std::min(cap - 1, j.size());
            std::memcpy(json, j.data(), n);
            json[n] = 0;
        }
    });
}

int shm_boot_get_split(const shm_boot *b, int *g1) {
    return guard([&] {
        if (!b || !g1) throw Error("null argument");
        for (int i = 0; i < 6; i++) g1[i] = b->b->params().bsgs_g1[i];
    });
}

int shm_boot_set_split(shm_boot *b, const int *g1) {
    return guard([&] {
        if (!b || !g1) throw Error("null argument");
        b->b->set_split(g1);
    });
}

int shm_boot_capture(shm_boot *b, const shm_ct *in, uint32_t members, shm_ct **out, shm_host_graph **graph) {
    return guard([&] {
        if (!b) throw Error("null bootstrapper");
        if (!graph || !out) throw Error("null output handle");
        if (members) b->h->use_shared(members);
        Ciphertext o;
        std::unique_ptr<Graph> g = b->b->capture(C(in), members, o);
        *graph = new shm_host_graph{std::move(g)};
        put(out, std::move(o));
    });
}

int shm_host_graph_launch(shm_host_graph *g) {
    return guard([&] {
        if (!g) throw Error("null graph");
        g->g->launch();
    });
}

uint64_t shm_host_graph_kernels(const shm_host_graph *g) { return g ? g->g->kernels() : 0; }

void shm_host_graph_destroy(shm_host_graph *g) { delete g; }

int shm_server_create(shm_host *h, shm_boot *boot, size_t hbm_budget_bytes, uint32_t slots, uint32_t max_merge,
                      shm_server **out) {
    return guard([&] {
        auto &hh = H(h);
        if (!out) throw Error("null output handle");
        *out = new shm_server{std::unique_ptr<Server>(
            new Server(*hh.ev, boot ? boot->b.get() : nullptr, &hh.shared, hbm_budget_bytes, slots, max_merge))};
    });
}

void shm_server_destroy(shm_server *s) { delete s; }

namespace {
Server &SV(shm_server *s) {
    if (!s || !s->s) throw Error("null server handle");
    return *s->s;
}
Ciphertext take(shm_ct *ct) {
    if (!ct) throw Error("null ciphertext handle");
    Ciphertext c = std::move(ct->ct);
    delete ct;
    return c;
}
}  // namespace

int shm_server_submit_rotate(shm_server *s, shm_ct *ct, int step, uint64_t *job) {
    return guard([&] {
        Server &sv = SV(s);
        *job = sv.submit_rotate(take(ct), step);
    });
}

int shm_server_submit_matmul(shm_server *s, shm_ct *X, const int64_t *W, uint32_t n_out, double w_scale,
                             uint64_t *job) {
    return guard([&] {
        Server &sv = SV(s);
        if (!X || !W) throw Error("null argument");
        const size_t n_in = X->ct.count;
        *job = sv.submit_matmul(take(X), std::vector<int64_t>(W, W + n_in * n_out), n_out, w_scale);
    });
}

int shm_server_submit_bootstrap(shm_server *s, shm_ct *ct, uint32_t members, uint64_t *job) {
    return guard([&] {
        Server &sv = SV(s);
        *job = sv.submit_bootstrap(take(ct), members);
    });
}

int shm_server_wait(shm_server *s, uint64_t job, shm_ct **out, double *times, uint32_t *batched_with) {
    return guard([&] {
        ServeResult r = SV(s).wait(job);
        if (times) {
            times[0] = r.t_submit;
            times[1] = r.t_start;
            times[2] = r.t_end;
        }
        if (batched_with) *batched_with = r.batched_with;
        if (!r.error.empty()) throw Error(r.error);
        put(out, std::move(r.output));
    });
}

int shm_server_set_paused(shm_server *s, int paused) {
    return guard([&] { SV(s).set_paused(paused != 0); });
}

int shm_server_stats(const shm_server *s, size_t *budget, size_t *peak_admitted, uint32_t *max_inflight,
                     uint64_t *batches, uint64_t *jobs) {
    return guard([&] {
        ServeStats st = SV(const_cast<shm_server *>(s)).stats();
        if (budget) *budget = st.budget;
        if (peak_admitted) *peak_admitted = st.peak_admitted;
        if (max_inflight) *max_inflight = st.max_inflight;
        if (batches) *batches = st.batches;
        if (jobs) *jobs = st.jobs;
    });
}

double shm_slot_transform_selfcheck(uint32_t log_slots) {
    try {
        return slot_transform_selfcheck(log_slots);
    } catch (...) {
        return -1.0;
    }
}

}  // extern "C"
