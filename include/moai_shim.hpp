// Source-compatibility layer for MOAI driver code: the reference's moai:: host classes
// (src/include/source/ckks_evaluator_parallel.cuh:13-680), the PhantomFHE types and
// calls they take (EncryptionParameters, CoeffModulus::Create, PhantomContext,
// PhantomSecretKey, PhantomPublicKey, PhantomRelinKey, PhantomGaloisKey,
// PhantomCiphertext, PhantomPlaintext, PhantomCKKSEncoder), the packing helpers
// batch_input / bias_vec (matrix_mul/Batch_encode_encrypt.cuh) and
// ct_pt_matrix_mul_wo_pre (matrix_mul/Ct_pt_matrix_mul.cuh:18-185), over the C++ host
// library of include/shmoai/host.hpp.  Driver code written against those names compiles
// against this header and links libshmoai_host.so (GPU) or the oracle build of it (CPU).
//
// Header only, plain C++17 (no CUDA compiler needed).  Differences a driver can see:
//   * every ciphertext is NTT form (transform_to_ntt / transform_from_ntt are not offered);
//   * scales are tracked exactly; scale() is still a mutable reference, as drivers reset it;
//   * the reference's streams are accepted and ignored: each context has one stream;
//   * a plaintext made by encode(double) is the constant round(value * scale), which is what
//     the reference's FFT of a constant slot vector produces;
//   * ct_pt_matrix_mul_wo_pre runs as one batched exact contraction on the tensor cores
//     instead of 2 * col_W * row_W multiply_plain / add_inplace calls; the output is the same
//     (bit for bit on the same inputs, the weights encoded at the inputs' scale).
#pragma once

#include <cmath>
#include <complex>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "shmoai/host.hpp"

namespace phantom {

enum class scheme_type : uint8_t { none = 0, bfv = 1, ckks = 2, bgv = 3 };

// a prime of the chain; the value is known once a context made it (CoeffModulus::Create
// records only the bit size, as the context generates the primes)
struct Modulus {
    int bit_count = 0;
    uint64_t value_ = 0;
    uint64_t value() const { return value_; }
};

struct CoeffModulus {
    static std::vector<Modulus> Create(size_t poly_modulus_degree, const std::vector<int> &bit_sizes) {
        if (poly_modulus_degree < 2 || (poly_modulus_degree & (poly_modulus_degree - 1)))
            throw std::invalid_argument("poly_modulus_degree must be a power of two");
        std::vector<Modulus> out;
        for (int b : bit_sizes) out.push_back(Modulus{b, 0});
        return out;
    }
};

class EncryptionParameters {
   public:
    explicit EncryptionParameters(scheme_type s = scheme_type::ckks) : scheme_(s) {
        if (s != scheme_type::ckks) throw std::invalid_argument("only CKKS is provided");
    }
    void set_poly_modulus_degree(size_t n) { n_ = n; }
    void set_coeff_modulus(const std::vector<Modulus> &m) { mod_ = m; }
    // the last special_modulus_size primes are the key-switching primes P (default 1)
    void set_special_modulus_size(size_t k) { special_ = k; }
    // full packing only: sparse_slots must be 0 or N / 2
    void set_sparse_slots(size_t s) { sparse_ = s; }
    // the primes a context generated for the bit sizes
    void set_coeff_values(const std::vector<uint64_t> &v) {
        for (size_t i = 0; i < mod_.size() && i < v.size(); i++) mod_[i].value_ = v[i];
    }
    size_t poly_modulus_degree() const { return n_; }
    const std::vector<Modulus> &coeff_modulus() const { return mod_; }
    size_t special_modulus_size() const { return special_; }
    size_t sparse_slots() const { return sparse_; }
    scheme_type scheme() const { return scheme_; }

   private:
    scheme_type scheme_;
    size_t n_ = 0, special_ = 1, sparse_ = 0;
    std::vector<Modulus> mod_;
};

namespace util {
// the reference's stream handle; this layer runs every call on its context's stream
struct cuda_stream_wrapper {};
}  // namespace util

}  // namespace phantom

// ---------------------------------------------------------------- PhantomFHE types

class PhantomContext {
   public:
    explicit PhantomContext(const phantom::EncryptionParameters &p) : parms_(p) {
        const size_t n = p.poly_modulus_degree();
        uint32_t log_n = 0;
        while ((size_t(1) << log_n) < n) log_n++;
        if (p.sparse_slots() && p.sparse_slots() != n / 2)
            throw std::invalid_argument("sparse slot packing is not provided: use N / 2 slots");
        std::vector<int> bits;
        for (auto &m : p.coeff_modulus()) bits.push_back(m.bit_count);
        ctx_ = std::make_unique<shmoai::Context>(log_n, bits, (uint32_t)p.special_modulus_size());
        enc_ = std::make_unique<shmoai::Encoder>(*ctx_);
        ev_ = std::make_unique<shmoai::Evaluator>(*ctx_, *enc_);
        parms_.set_coeff_values(ctx_->primes);
    }
    const phantom::EncryptionParameters &parms() const { return parms_; }
    shmoai::Context &ctx() const { return *ctx_; }
    shmoai::Encoder &encoder() const { return *enc_; }
    shmoai::Evaluator &evaluator() const { return *ev_; }
    // chain index of a ciphertext with L primes (context.cu:148-174) and back
    size_t chain_index_of(uint32_t L) const { return ctx_->chain_index(L); }
    uint32_t limbs_of(size_t chain_index) const {
        if (chain_index < 1 || chain_index > ctx_->nq) throw std::invalid_argument("chain index out of range");
        return (uint32_t)(ctx_->nq - chain_index + 1);
    }

   private:
    phantom::EncryptionParameters parms_;
    std::unique_ptr<shmoai::Context> ctx_;
    std::unique_ptr<shmoai::Encoder> enc_;
    std::unique_ptr<shmoai::Evaluator> ev_;
};

class PhantomPlaintext {
   public:
    PhantomPlaintext() = default;
    PhantomPlaintext(const PhantomPlaintext &o) { *this = o; }
    PhantomPlaintext &operator=(const PhantomPlaintext &o) {
        if (this != &o) {
            ctx = o.ctx;
            pt.L = o.pt.L;
            pt.scale = o.pt.scale;
            pt.data = o.pt.data.words() ? o.pt.data.clone() : shmoai::DeviceBuffer();
        }
        return *this;
    }
    PhantomPlaintext(PhantomPlaintext &&) = default;
    PhantomPlaintext &operator=(PhantomPlaintext &&) = default;

    double &scale() { return pt.scale; }
    double scale() const { return pt.scale; }
    size_t chain_index() const { return ctx ? ctx->chain_index_of(pt.L) : 0; }
    size_t params_id() const { return chain_index(); }
    size_t coeff_modulus_size() const { return pt.L; }
    uint64_t *data() const { return pt.data.data(); }

    const PhantomContext *ctx = nullptr;
    shmoai::Plaintext pt;
};

class PhantomCiphertext {
   public:
    PhantomCiphertext() = default;
    PhantomCiphertext(const PhantomCiphertext &o) { *this = o; }  // a device copy, as the reference's
    PhantomCiphertext &operator=(const PhantomCiphertext &o) {
        if (this != &o) {
            ctx = o.ctx;
            ct.count = o.ct.count;
            ct.size = o.ct.size;
            ct.L = o.ct.L;
            ct.scale_ = o.ct.scale_;
            ct.shared = o.ct.shared;
            ct.data = o.ct.data.words() ? o.ct.data.clone() : shmoai::DeviceBuffer();
        }
        return *this;
    }
    PhantomCiphertext(PhantomCiphertext &&) = default;
    PhantomCiphertext &operator=(PhantomCiphertext &&) = default;

    double &scale() { return ct.scale_; }
    double scale() const { return ct.scale_; }
    size_t chain_index() const { return ctx ? ctx->chain_index_of(ct.L) : 0; }
    size_t params_id() const { return chain_index(); }
    size_t coeff_modulus_size() const { return ct.L; }
    size_t size() const { return ct.size; }
    size_t poly_modulus_degree() const { return ctx ? ctx->ctx().n : 0; }
    bool is_ntt_form() const { return true; }
    uint64_t *data() const { return ct.data.data(); }

    const PhantomContext *ctx = nullptr;
    shmoai::Ciphertext ct;  // one ciphertext (count 1)
};

struct PhantomRelinKey {
    shmoai::DeviceBuffer key;  // [dnum][2][QP][N]
};

struct PhantomGaloisKey {
    std::map<uint32_t, shmoai::DeviceBuffer> keys;  // Galois element -> [dnum][2][QP][N]
};

struct PhantomPublicKey {
    std::shared_ptr<shmoai::PublicEncryptor> enc;  // holds pk = (e - a s, a) over QP
};

class PhantomSecretKey {
   public:
    // a ternary secret of Hamming weight h (the MOAI setting is 192), deterministic in seed
    explicit PhantomSecretKey(const PhantomContext &c, uint32_t hamming_weight = 192, uint64_t seed = 0x5EED)
        : ctx_(&c), kg_(std::make_unique<shmoai::KeyGenerator>(c.ctx(), hamming_weight, seed)) {}
    PhantomPublicKey gen_publickey(const PhantomContext &) const {
        return PhantomPublicKey{std::make_shared<shmoai::PublicEncryptor>(ctx_->ctx(), kg_->public_key(),
                                                                          0xE0C0 + ++pub_count_)};
    }
    PhantomRelinKey gen_relinkey(const PhantomContext &) const { return PhantomRelinKey{kg_->relin_key()}; }
    PhantomGaloisKey create_galois_keys_from_steps(const PhantomContext &, const std::vector<int> &steps) const {
        PhantomGaloisKey g;
        for (int s : steps) {
            const uint32_t e = s == 0 ? 2 * ctx_->ctx().n - 1 : ctx_->evaluator().galois_elt(s);
            if (!g.keys.count(e)) g.keys.emplace(e, kg_->galois_key(e));
        }
        return g;
    }
    PhantomGaloisKey create_galois_keys_from_elts(const PhantomContext &, const std::vector<uint32_t> &elts) const {
        PhantomGaloisKey g;
        for (uint32_t e : elts)
            if (!g.keys.count(e)) g.keys.emplace(e, kg_->galois_key(e));
        return g;
    }
    // c0 + c1 s at the ciphertext's level (ckks_decrypt, secretkey.cu:725-765)
    void decrypt(const PhantomContext &c, const PhantomCiphertext &ct, PhantomPlaintext &out) const {
        if (ct.ct.size != 2 || ct.ct.count != 1) throw std::invalid_argument("decrypt: one size-2 ciphertext");
        const shmoai::Context &x = c.ctx();
        const uint32_t L = ct.ct.L;
        const size_t ln = (size_t)L * x.n;
        out.ctx = &c;
        out.pt.L = L;
        out.pt.scale = ct.ct.scale_;
        out.pt.data = shmoai::DeviceBuffer(x, ln);
        shmoai::DeviceBuffer t(x, ln);
        x.check(shm_multiply_plain(x.handle(), ct.ct.data.data() + ln, kg_->secret().data(), t.data(), 1, L,
                                   x.stream()));
        x.check(shm_add(x.handle(), ct.ct.data.data(), t.data(), out.pt.data.data(), 1, L, x.stream()));
    }
    shmoai::KeyGenerator &generator() const { return *kg_; }

   private:
    const PhantomContext *ctx_;
    std::unique_ptr<shmoai::KeyGenerator> kg_;
    mutable uint64_t pub_count_ = 0;
};

class PhantomCKKSEncoder {
   public:
    explicit PhantomCKKSEncoder(const PhantomContext &c) : ctx_(&c) {}
    size_t slot_count() const { return ctx_->ctx().n / 2; }
    const PhantomContext &context() const { return *ctx_; }
    // PhantomCKKSEncoder::encode (thirdparty/phantom-fhe/include/ckks.h:84-95): slot values (double or
    // complex) at a chain index
    template <class T>
    void encode(const PhantomContext &c, const std::vector<T> &values, double scale, PhantomPlaintext &dest,
                size_t chain_index = 1, const phantom::util::cuda_stream_wrapper & = {}) const {
        if (values.size() > slot_count()) throw std::invalid_argument("values_size is too large");
        std::vector<std::complex<double>> z(values.begin(), values.end());
        dest.ctx = &c;
        dest.pt = c.encoder().encode(z, c.limbs_of(chain_index), scale);
    }

   private:
    const PhantomContext *ctx_;
};

namespace moai {

using std::vector;
using cplx = std::complex<double>;
using phantom::util::cuda_stream_wrapper;

namespace detail {
inline PhantomCiphertext wrap(const PhantomContext *c, shmoai::Ciphertext &&ct) {
    PhantomCiphertext out;
    out.ctx = c;
    out.ct = std::move(ct);
    return out;
}
inline const cuda_stream_wrapper &no_stream() {
    static cuda_stream_wrapper s;
    return s;
}
}  // namespace detail

class Encoder {
   public:
    Encoder() = default;
    Encoder(PhantomContext *context, PhantomCKKSEncoder *encoder) : context_(context), encoder_(encoder) {}
    size_t slot_count() const { return encoder_->slot_count(); }
    void reset_sparse_slots() {}

    void encode(vector<double> values, size_t chain_index, double scale, PhantomPlaintext &plain,
                const cuda_stream_wrapper & = detail::no_stream()) {
        if (values.size() == 1) return encode(values[0], chain_index, scale, plain);
        vector<cplx> z(values.begin(), values.end());
        encode_slots(z, chain_index, scale, plain);
    }
    void encode(vector<double> values, double scale, PhantomPlaintext &plain,
                const cuda_stream_wrapper &s = detail::no_stream()) {
        encode(std::move(values), 1, scale, plain, s);
    }
    void encode(vector<cplx> values, double scale, PhantomPlaintext &plain,
                const cuda_stream_wrapper & = detail::no_stream()) {
        if (values.size() == 1) return encode(values[0], scale, plain);
        encode_slots(values, 1, scale, plain);
    }
    // a value in every slot: the constant polynomial round(value * scale)
    void encode(double value, size_t chain_index, double scale, PhantomPlaintext &plain,
                const cuda_stream_wrapper & = detail::no_stream()) {
        plain.ctx = context_;
        plain.pt = context_->encoder().encode(value, context_->limbs_of(chain_index), scale);
    }
    void encode(double value, double scale, PhantomPlaintext &plain, const cuda_stream_wrapper &s = detail::no_stream()) {
        encode(value, 1, scale, plain, s);
    }
    void encode(cplx value, double scale, PhantomPlaintext &plain, const cuda_stream_wrapper & = detail::no_stream()) {
        encode_slots(vector<cplx>(slot_count(), value), 1, scale, plain);
    }

    template <typename T>
    void decode(const PhantomPlaintext &plain, vector<T> &values, const cuda_stream_wrapper & = detail::no_stream()) {
        const shmoai::Context &x = context_->ctx();
        // limb 0 to coefficient form, centred: the message while |m| < q0 / 2
        shmoai::DeviceBuffer l0(x, x.n);
        x.check(shm_drop_limbs(x.handle(), plain.pt.data.data(), l0.data(), 1, plain.pt.L, 1, x.stream()));
        x.check(shm_ntt_inverse(x.handle(), l0.data(), 1, 1, x.stream()));
        std::vector<uint64_t> r(x.n);
        x.check(shm_memcpy(x.handle(), r.data(), l0.data(), x.n * 8, SHM_COPY_D2H, x.stream()));
        x.synchronize();
        const uint64_t q0 = x.primes[0];
        std::vector<double> c(x.n);
        for (size_t k = 0; k < x.n; k++) c[k] = r[k] > q0 / 2 ? -(double)(q0 - r[k]) : (double)r[k];
        std::vector<cplx> z = context_->encoder().decode(c, plain.pt.scale);
        values.resize(z.size());
        for (size_t j = 0; j < z.size(); j++) assign(values[j], z[j]);
    }

   private:
    static void assign(double &d, const cplx &z) { d = z.real(); }
    static void assign(cplx &d, const cplx &z) { d = z; }
    void encode_slots(const vector<cplx> &z, size_t chain_index, double scale, PhantomPlaintext &plain) {
        if (z.size() > slot_count()) throw std::invalid_argument("values_size is too large");
        plain.ctx = context_;
        plain.pt = context_->encoder().encode(z, context_->limbs_of(chain_index), scale);
    }
    PhantomContext *context_ = nullptr;
    PhantomCKKSEncoder *encoder_ = nullptr;
};

class Encryptor {
   public:
    Encryptor() = default;
    Encryptor(PhantomContext *context, PhantomPublicKey *pk) : context_(context), pk_(pk) {}
    void encrypt(PhantomPlaintext &plain, PhantomCiphertext &ct, const cuda_stream_wrapper & = detail::no_stream()) {
        ct = detail::wrap(context_, pk_->enc->encrypt(plain.pt));
    }

   private:
    PhantomContext *context_ = nullptr;
    PhantomPublicKey *pk_ = nullptr;
};

class Decryptor {
   public:
    Decryptor() = default;
    Decryptor(PhantomContext *context, PhantomSecretKey *sk) : context_(context), sk_(sk) {}
    void decrypt(PhantomCiphertext &ct, PhantomPlaintext &plain, const cuda_stream_wrapper & = detail::no_stream()) {
        sk_->decrypt(*context_, ct, plain);
    }
    void create_galois_keys_from_steps(vector<int> &steps, PhantomGaloisKey &keys,
                                       const cuda_stream_wrapper & = detail::no_stream()) {
        keys = sk_->create_galois_keys_from_steps(*context_, steps);
    }
    void create_galois_keys_from_elts(vector<uint32_t> &elts, PhantomGaloisKey &keys,
                                      const cuda_stream_wrapper & = detail::no_stream()) {
        keys = sk_->create_galois_keys_from_elts(*context_, elts);
    }

   private:
    PhantomContext *context_ = nullptr;
    PhantomSecretKey *sk_ = nullptr;
};

// moai::Evaluator (ckks_evaluator_parallel.cuh:150-562) on single ciphertexts
class Evaluator {
   public:
    Evaluator() = default;
    Evaluator(PhantomContext *context, PhantomCKKSEncoder *encoder) : context_(context), encoder_(encoder) {}

    using CS = cuda_stream_wrapper;
    void multiply_plain(PhantomCiphertext &ct, PhantomPlaintext &plain, PhantomCiphertext &dest,
                        const CS & = detail::no_stream()) {
        dest = detail::wrap(context_, ev().multiply_plain(ct.ct, level(plain, ct.ct.L)));
    }
    void multiply_plain_inplace(PhantomCiphertext &ct, PhantomPlaintext &plain, const CS &s = detail::no_stream()) {
        multiply_plain(ct, plain, ct, s);
    }
    void add(PhantomCiphertext &a, const PhantomCiphertext &b, PhantomCiphertext &dest, const CS & = detail::no_stream()) {
        dest = detail::wrap(context_, ev().add(a.ct, b.ct));
    }
    void add_inplace(PhantomCiphertext &a, const PhantomCiphertext &b, const CS &s = detail::no_stream()) {
        add(a, b, a, s);
    }
    void sub(PhantomCiphertext &a, const PhantomCiphertext &b, PhantomCiphertext &dest, const CS & = detail::no_stream()) {
        dest = detail::wrap(context_, ev().sub(a.ct, b.ct));
    }
    void sub_inplace(PhantomCiphertext &a, const PhantomCiphertext &b, const CS &s = detail::no_stream()) {
        sub(a, b, a, s);
    }
    void negate_inplace(PhantomCiphertext &a, const CS & = detail::no_stream()) {
        a = detail::wrap(context_, ev().negate(a.ct));
    }
    void add_plain(PhantomCiphertext &ct, PhantomPlaintext &plain, PhantomCiphertext &dest,
                   const CS & = detail::no_stream()) {
        dest = ct;
        add_plain_inplace(dest, plain);
    }
    void add_plain_inplace(PhantomCiphertext &ct, PhantomPlaintext &plain, const CS & = detail::no_stream()) {
        const shmoai::Plaintext &p = level(plain, ct.ct.L);
        if (!shmoai::Evaluator::same_scale(ct.ct.scale_, p.scale, 1e-6))
            throw std::invalid_argument("add_plain: scale mismatch");
        const shmoai::Context &x = context_->ctx();
        x.check(shm_add(x.handle(), ct.ct.data.data(), p.data.data(), ct.ct.data.data(), 1, ct.ct.L, x.stream()));
    }
    void multiply(PhantomCiphertext &a, const PhantomCiphertext &b, PhantomCiphertext &dest,
                  const CS & = detail::no_stream()) {
        dest = detail::wrap(context_, ev().multiply_lazy(a.ct, b.ct));
    }
    void multiply_inplace(PhantomCiphertext &a, const PhantomCiphertext &b, const CS &s = detail::no_stream()) {
        multiply(a, b, a, s);
    }
    void square(PhantomCiphertext &a, PhantomCiphertext &dest, const CS &s = detail::no_stream()) { multiply(a, a, dest, s); }
    void square_inplace(PhantomCiphertext &a, const CS &s = detail::no_stream()) { multiply(a, a, a, s); }
    void relinearize_inplace(PhantomCiphertext &ct, const PhantomRelinKey &rk, const CS & = detail::no_stream()) {
        auto &e = ev();
        e.relin_key = &rk.key;
        ct = detail::wrap(context_, e.relinearize(ct.ct));
    }
    void rescale_to_next(const PhantomCiphertext &ct, PhantomCiphertext &dest, const CS & = detail::no_stream()) {
        dest = detail::wrap(context_, ev().rescale_to_next(ct.ct));
    }
    void rescale_to_next_inplace(PhantomCiphertext &ct, const CS &s = detail::no_stream()) { rescale_to_next(ct, ct, s); }
    void mod_switch_to_inplace(PhantomCiphertext &ct, size_t chain_index, const CS & = detail::no_stream()) {
        ct = detail::wrap(context_, ev().mod_switch_to(ct.ct, context_->limbs_of(chain_index)));
    }
    void mod_switch_to_next_inplace(PhantomCiphertext &ct, const CS & = detail::no_stream()) {
        ct = detail::wrap(context_, ev().mod_switch_to(ct.ct, ct.ct.L - 1));
    }
    void mod_switch_to_inplace(PhantomPlaintext &pt, size_t chain_index, const CS & = detail::no_stream()) {
        const uint32_t L = context_->limbs_of(chain_index);
        if (L != pt.pt.L) pt.pt = level(pt, L);
    }
    void rotate_vector(PhantomCiphertext &ct, int steps, PhantomGaloisKey &gk, PhantomCiphertext &dest,
                       const CS & = detail::no_stream()) {
        auto &e = ev();
        e.galois_keys = &gk.keys;
        dest = detail::wrap(context_, e.rotate_vector(ct.ct, steps));
    }
    void rotate_vector_inplace(PhantomCiphertext &ct, int steps, PhantomGaloisKey &gk, const CS &s = detail::no_stream()) {
        rotate_vector(ct, steps, gk, ct, s);
    }
    void complex_conjugate(PhantomCiphertext &ct, PhantomGaloisKey &gk, PhantomCiphertext &dest,
                           const CS & = detail::no_stream()) {
        auto &e = ev();
        e.galois_keys = &gk.keys;
        dest = detail::wrap(context_, e.complex_conjugate(ct.ct));
    }
    // value encoded at the ciphertext's level and scale, then multiply_plain (scale squared), as the
    // reference's multiply_const
    void multiply_const(const PhantomCiphertext &ct, double value, PhantomCiphertext &dest,
                        const CS & = detail::no_stream()) {
        shmoai::Plaintext p = context_->encoder().encode(value, ct.ct.L, ct.ct.scale_);
        dest = detail::wrap(context_, ev().multiply_plain(ct.ct, p));
    }
    void multiply_const_inplace(PhantomCiphertext &ct, double value, const CS &s = detail::no_stream()) {
        multiply_const(ct, value, ct, s);
    }
    void add_const(PhantomCiphertext &ct, double value, PhantomCiphertext &dest, const CS & = detail::no_stream()) {
        dest = detail::wrap(context_, ev().add_const(ct.ct, value));
    }
    void add_const_inplace(PhantomCiphertext &ct, double value, const CS &s = detail::no_stream()) {
        add_const(ct, value, ct, s);
    }
    void double_inplace(PhantomCiphertext &ct, const CS & = detail::no_stream()) {
        ct = detail::wrap(context_, ev().add(ct.ct, ct.ct));
    }

   private:
    shmoai::Evaluator &ev() const { return context_->evaluator(); }
    // a plaintext at L primes (its first L limbs)
    shmoai::Plaintext level(const PhantomPlaintext &p, uint32_t L) const {
        if (p.pt.L < L) throw std::invalid_argument("plaintext below the ciphertext's level");
        const shmoai::Context &x = context_->ctx();
        shmoai::Plaintext out;
        out.L = L;
        out.scale = p.pt.scale;
        out.data = shmoai::DeviceBuffer(x, (size_t)L * x.n);
        x.check(shm_drop_limbs(x.handle(), p.pt.data.data(), out.data.data(), 1, p.pt.L, L, x.stream()));
        return out;
    }
    PhantomContext *context_ = nullptr;
    PhantomCKKSEncoder *encoder_ = nullptr;
};

// moai::CKKSEvaluator (ckks_evaluator_parallel.cuh:600-680): the component classes and the
// non-linear helpers that the host library provides (exp, inverse, invert_sqrt)
class CKKSEvaluator {
   public:
    PhantomContext *context;
    PhantomRelinKey *relin_keys;
    PhantomGaloisKey *galois_keys;
    std::vector<uint32_t> galois_elts;
    Encoder encoder;
    Encryptor encryptor;
    Evaluator evaluator;
    Decryptor decryptor;
    size_t degree;
    double scale;
    size_t slot_count;

    CKKSEvaluator(PhantomContext *ctx, PhantomPublicKey *pk, PhantomSecretKey *sk, PhantomCKKSEncoder *enc,
                  PhantomRelinKey *rk, PhantomGaloisKey *gk, double scale_, std::vector<uint32_t> elts = {})
        : context(ctx), relin_keys(rk), galois_keys(gk), galois_elts(std::move(elts)), encoder(ctx, enc),
          encryptor(ctx, pk), evaluator(ctx, enc), decryptor(ctx, sk), degree(enc->slot_count() * 2),
          scale(scale_), slot_count(enc->slot_count()) {}

    PhantomCiphertext exp(PhantomCiphertext x) { return apply(x, [](const shmoai::Evaluator &e, const shmoai::Ciphertext &c) {
        return shmoai::exp_approx(e, c);
    }); }
    PhantomCiphertext inverse(PhantomCiphertext x, int iter = 4) {
        return apply(x, [iter](const shmoai::Evaluator &e, const shmoai::Ciphertext &c) {
            return shmoai::inverse_approx(e, c, iter);
        });
    }
    PhantomCiphertext invert_sqrt(PhantomCiphertext x, int d_newt = 20, int d_gold = 1) {
        return apply(x, [d_newt, d_gold](const shmoai::Evaluator &e, const shmoai::Ciphertext &c) {
            return shmoai::inv_sqrt_approx(e, c, d_newt, d_gold);
        });
    }

   private:
    template <typename F>
    PhantomCiphertext apply(const PhantomCiphertext &x, F f) {
        shmoai::Evaluator &e = context->evaluator();
        e.relin_key = &relin_keys->key;
        e.galois_keys = galois_keys ? &galois_keys->keys : nullptr;
        return detail::wrap(context, f(e, x.ct));
    }
};

}  // namespace moai

// ---------------------------------------------------------------- MOAI driver helpers

// batch_input (Batch_encode_encrypt.cuh:12-43): X[j][k][i] of num_X inputs of num_row x num_col
// -> num_col ciphertexts, column-interleaved, encrypted with the public key at the top level
inline std::vector<PhantomCiphertext> batch_input(const std::vector<std::vector<std::vector<double>>> &X, int num_X,
                                                  int num_row, int num_col, double scale, PhantomContext &context,
                                                  PhantomPublicKey &pk) {
    std::vector<double> flat((size_t)num_X * num_row * num_col);
    for (int j = 0; j < num_X; j++)
        for (int k = 0; k < num_row; k++)
            for (int i = 0; i < num_col; i++) flat[((size_t)j * num_row + k) * num_col + i] = X[j][k][i];
    shmoai::Ciphertext all = shmoai::batch_input(*pk.enc, flat, (uint32_t)num_X, (uint32_t)num_row, (uint32_t)num_col,
                                                 scale, context.ctx().nq);
    std::vector<PhantomCiphertext> out;
    for (int i = 0; i < num_col; i++)
        out.push_back(moai::detail::wrap(&context, context.evaluator().slice(all, (uint32_t)i, 1)));
    return out;
}

inline std::vector<int> bias_vec(const std::vector<int> &lengths, int num_X, int num_row) {
    return shmoai::bias_vec(lengths, (uint32_t)num_X, (uint32_t)num_row);
}

// ct_pt_matrix_mul_wo_pre (Ct_pt_matrix_mul.cuh:18-185): output i = rescale(sum_j enc_X[j] * W[j][i])
// with every weight encoded as the constant round(W[j][i] * scale of enc_X[0]) and the output's scale
// reset to the input's, as the reference does; one batched exact contraction
inline std::vector<PhantomCiphertext> ct_pt_matrix_mul_wo_pre(std::vector<PhantomCiphertext> &enc_X,
                                                              const std::vector<std::vector<double>> &W, int col_X,
                                                              int col_W, int row_W, PhantomContext &context) {
    if (enc_X.empty() || col_W <= 0 || row_W <= 0 || col_X != row_W || (int)enc_X.size() < row_W ||
        (int)W.size() < row_W)
        throw std::invalid_argument("ct_pt_matrix_mul_wo_pre: bad dimensions");
    const double scale = enc_X[0].scale();
    shmoai::Evaluator &ev = context.evaluator();
    const shmoai::Context &x = context.ctx();
    // the inputs as one batch [row_W][2][L][N] (device copies)
    shmoai::Ciphertext X;
    X.count = (uint32_t)row_W;
    X.size = 2;
    X.L = enc_X[0].ct.L;
    X.scale_ = scale;
    const size_t words = 2 * (size_t)X.L * x.n;
    X.data = shmoai::DeviceBuffer(x, words * row_W);
    for (int j = 0; j < row_W; j++) {
        const shmoai::Ciphertext &c = enc_X[j].ct;
        if (c.count != 1 || c.size != 2 || c.L != X.L || !shmoai::Evaluator::same_scale(c.scale_, scale, 1e-6))
            throw std::invalid_argument("ct_pt_matrix_mul_wo_pre: inputs differ in level, size or scale");
        x.check(shm_memcpy(x.handle(), X.data.data() + j * words, c.data.data(), words * 8, SHM_COPY_D2D, x.stream()));
    }
    std::vector<int64_t> Wi((size_t)row_W * col_W);
    for (int j = 0; j < row_W; j++) {
        if ((int)W[j].size() < col_W) throw std::invalid_argument("ct_pt_matrix_mul_wo_pre: short W row");
        for (int i = 0; i < col_W; i++) Wi[(size_t)j * col_W + i] = (int64_t)std::llround(W[j][i] * scale);
    }
    shmoai::Ciphertext Y = ev.ctpt_matmul(X, Wi, (uint32_t)col_W, scale);
    std::vector<PhantomCiphertext> out;
    for (int i = 0; i < col_W; i++) {
        PhantomCiphertext c = moai::detail::wrap(&context, ev.slice(Y, (uint32_t)i, 1));
        c.scale() = scale;
        out.push_back(std::move(c));
    }
    return out;
}
