// Context, device buffers, the canonical-embedding encoder, key generation and
// symmetric encryption / decryption of the C++ host API (include/shmoai/host.hpp).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.hpp"

namespace shmoai {

// ------------------------------------------------------------------ Context

Context::Context(uint32_t log_n_, const std::vector<int> &bits, uint32_t n_special, int device, void *stream)
    : stream_(stream) {
    if (n_special >= bits.size()) throw Error("need at least one ciphertext prime");
    int rc = shm_context_create(&h_, log_n_, bits.data(), (uint32_t)(bits.size() - n_special), n_special, device);
    if (rc != SHM_OK) throw Error(std::string("shm_context_create: ") + shm_last_error());
    init();
}

Context::Context(uint32_t log_n_, const std::vector<uint64_t> &p, uint32_t n_special, int device, void *stream)
    : stream_(stream) {
    if (n_special >= p.size()) throw Error("need at least one ciphertext prime");
    int rc = shm_context_create_from_primes(&h_, log_n_, p.data(), (uint32_t)(p.size() - n_special), n_special,
                                            device);
    if (rc != SHM_OK) throw Error(std::string("shm_context_create_from_primes: ") + shm_last_error());
    init();
}

Context::Context(const Context &base, void *stream)
    : log_n(base.log_n), n(base.n), nq(base.nq), np(base.np), dnum(base.dnum), primes(base.primes), h_(base.h_),
      stream_(stream), owner_(false) {}

void Context::init() {
    check(shm_context_info(h_, &log_n, &nq, &np, &dnum));
    n = 1u << log_n;
    primes.resize(nq + np);
    check(shm_context_primes(h_, primes.data()));
}

Context::~Context() {
    if (h_) shm_synchronize(h_, stream_);
    if (h_ && owner_) shm_context_destroy(h_);
}

void Context::check(int rc) const {
    if (rc != SHM_OK) throw Error(shm_last_error(), rc);
}

void Context::synchronize() const { check(shm_synchronize(h_, stream_)); }

// ------------------------------------------------------------------ DeviceBuffer

DeviceBuffer::DeviceBuffer(const Context &c, size_t words) : ctx_(&c), words_(words) {
    void *p = nullptr;
    c.check(shm_malloc(c.handle(), words * 8, &p, c.stream()));
    p_ = static_cast<uint64_t *>(p);
}

DeviceBuffer::~DeviceBuffer() {
    if (p_ && ctx_) shm_free(ctx_->handle(), p_, ctx_->stream());
}

DeviceBuffer::DeviceBuffer(DeviceBuffer &&o) noexcept : ctx_(o.ctx_), p_(o.p_), words_(o.words_) {
    o.p_ = nullptr;
    o.words_ = 0;
}

DeviceBuffer &DeviceBuffer::operator=(DeviceBuffer &&o) noexcept {
    if (this != &o) {
        if (p_ && ctx_) shm_free(ctx_->handle(), p_, ctx_->stream());
        ctx_ = o.ctx_;
        p_ = o.p_;
        words_ = o.words_;
        o.p_ = nullptr;
        o.words_ = 0;
    }
    return *this;
}

DeviceBuffer DeviceBuffer::clone() const {
    if (!ctx_) return DeviceBuffer();
    DeviceBuffer d(*ctx_, words_);
    ctx_->check(shm_memcpy(ctx_->handle(), d.p_, p_, words_ * 8, SHM_COPY_D2D, ctx_->stream()));
    return d;
}

// ------------------------------------------------------------------ Encoder
//
// Slot j of m(X) (degree < N, N/2 slots) is m(omega_j) / scale with
// omega_j = exp(2 pi i 5^j / 2N), the slot order of the reference encoder
// (thirdparty/phantom-fhe/src/ckks.cu:20-87): X -> X^(5^s) rotates the slots left by s.
//   encode: m_k = round((2 scale / N) Re(sum_j z_j omega_j^-k)), one length-2N FFT;
//   decode: z_j = (sum_k m_k omega_j^k) / scale, one length-2N inverse FFT.

Encoder::Encoder(const Context &c) : c_(c) {
    const uint32_t M = 2 * c.n, slots = c.n / 2;
    exps_.resize(slots);
    uint64_t e = 1;
    for (uint32_t j = 0; j < slots; j++) {
        exps_[j] = (uint32_t)e;
        e = (e * 5) % M;
    }
    roots_.resize(M);
    for (uint32_t k = 0; k < M; k++) {
        const double ang = 2.0 * M_PI * (double)k / (double)M;
        roots_[k] = cplx(std::cos(ang), std::sin(ang));
    }
}

// radix-2 decimation in time; forward X_k = sum_j a_j e^{-2 pi i jk/M}, inverse without 1/M
void Encoder::fft(std::vector<cplx> &a, bool inverse) const {
    const size_t M = a.size();
    for (size_t i = 1, j = 0; i < M; i++) {
        size_t bit = M >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= M; len <<= 1) {
        const size_t stride = M / len, half = len / 2;
        for (size_t i = 0; i < M; i += len)
            for (size_t k = 0; k < half; k++) {
                cplx w = roots_[k * stride];
                if (!inverse) w = std::conj(w);
                const cplx u = a[i + k], v = a[i + k + half] * w;
                a[i + k] = u + v;
                a[i + k + half] = u - v;
            }
    }
}

std::vector<double> Encoder::encode_float(const cplx *z, size_t len, double scale) const {
    const uint32_t N = c_.n, M = 2 * N, slots = N / 2;
    if (len > slots) throw Error("more values than slots");
    std::vector<cplx> A(M, cplx(0, 0));
    for (size_t j = 0; j < len; j++) A[exps_[j]] = z[j];
    fft(A, false);
    std::vector<double> out(N);
    const double f = 2.0 * scale / (double)N;
    for (uint32_t k = 0; k < N; k++) out[k] = f * A[k].real();
    return out;
}

void Encoder::encode_rows(const std::vector<std::vector<cplx>> &z, double scale, uint64_t *coeffs) const {
    const uint32_t rows = (uint32_t)z.size(), slots = c_.n / 2;
    size_t nv = 0;
    for (auto &r : z) nv = std::max(nv, r.size());
    if (nv > slots) throw Error("more values than slots");
    shm_context *h = c_.handle();
    DeviceBuffer dre, dim;
    if (nv) {
        std::vector<double> re(rows * nv, 0.0), im(rows * nv, 0.0);  // shorter rows padded with zero slots
        for (uint32_t i = 0; i < rows; i++)
            for (size_t j = 0; j < z[i].size(); j++) {
                re[i * nv + j] = z[i][j].real();
                im[i * nv + j] = z[i][j].imag();
            }
        dre = DeviceBuffer(c_, re.size());
        dim = DeviceBuffer(c_, im.size());
        c_.check(shm_memcpy(h, dre.data(), re.data(), re.size() * 8, SHM_COPY_H2D, c_.stream()));
        c_.check(shm_memcpy(h, dim.data(), im.data(), im.size() * 8, SHM_COPY_H2D, c_.stream()));
    }
    DeviceBuffer ws(c_, shm_encode_workspace_bytes(h, rows) / 8 + 1);
    c_.check(shm_encode(h, reinterpret_cast<const double *>(dre.data()), reinterpret_cast<const double *>(dim.data()),
                        rows, (uint32_t)nv, scale, reinterpret_cast<int64_t *>(coeffs), ws.data(), ws.words() * 8,
                        c_.stream()));
}

std::vector<int64_t> Encoder::encode_coeffs(const cplx *z, size_t len, double scale) const {
    DeviceBuffer d(c_, c_.n);
    encode_rows({std::vector<cplx>(z, z + len)}, scale, d.data());
    std::vector<int64_t> out(c_.n);
    c_.check(shm_memcpy(c_.handle(), out.data(), d.data(), c_.n * 8, SHM_COPY_D2H, c_.stream()));
    return out;
}

void Encoder::lift(const uint64_t *coeffs, size_t n_polys, uint32_t L, uint64_t *out) const {
    c_.check(shm_lift_signed(c_.handle(), reinterpret_cast<const int64_t *>(coeffs), out, (uint32_t)n_polys, L,
                             c_.stream()));
    c_.check(shm_ntt_forward(c_.handle(), out, (uint32_t)n_polys, L, c_.stream()));
}

void Encoder::lift_ext(const uint64_t *coeffs, size_t n_polys, uint32_t L, uint64_t *out) const {
    c_.check(shm_lift_signed_ext(c_.handle(), reinterpret_cast<const int64_t *>(coeffs), out, (uint32_t)n_polys, L,
                                 c_.stream()));
    c_.check(shm_ntt_forward_ext(c_.handle(), out, (uint32_t)n_polys, L, c_.stream()));
}

void Encoder::upload(const int64_t *coeffs, size_t n_polys, uint32_t L, uint64_t *out) const {
    DeviceBuffer tmp(c_, n_polys * c_.n);
    c_.check(shm_memcpy(c_.handle(), tmp.data(), coeffs, n_polys * c_.n * 8, SHM_COPY_H2D, c_.stream()));
    c_.check(shm_lift_signed(c_.handle(), reinterpret_cast<const int64_t *>(tmp.data()), out, (uint32_t)n_polys, L,
                             c_.stream()));
    c_.check(shm_ntt_forward(c_.handle(), out, (uint32_t)n_polys, L, c_.stream()));
}

void Encoder::upload_ext(const int64_t *coeffs, size_t n_polys, uint32_t L, uint64_t *out) const {
    DeviceBuffer tmp(c_, n_polys * c_.n);
    c_.check(shm_memcpy(c_.handle(), tmp.data(), coeffs, n_polys * c_.n * 8, SHM_COPY_H2D, c_.stream()));
    c_.check(shm_lift_signed_ext(c_.handle(), reinterpret_cast<const int64_t *>(tmp.data()), out, (uint32_t)n_polys,
                                 L, c_.stream()));
    c_.check(shm_ntt_forward_ext(c_.handle(), out, (uint32_t)n_polys, L, c_.stream()));
}

Plaintext Encoder::encode_ext(const std::vector<cplx> &z, uint32_t L, double scale) const {
    DeviceBuffer coeffs(c_, c_.n);
    encode_rows({z}, scale, coeffs.data());
    Plaintext p;
    p.data = DeviceBuffer(c_, (size_t)(L + c_.np) * c_.n);
    p.L = L;
    p.scale = scale;
    lift_ext(coeffs.data(), 1, L, p.data.data());
    return p;
}

Plaintext Encoder::encode(const std::vector<cplx> &z, uint32_t L, double scale) const {
    DeviceBuffer coeffs(c_, c_.n);
    encode_rows({z}, scale, coeffs.data());
    Plaintext p;
    p.data = DeviceBuffer(c_, (size_t)L * c_.n);
    p.L = L;
    p.scale = scale;
    lift(coeffs.data(), 1, L, p.data.data());
    return p;
}

Plaintext Encoder::encode(double value, uint32_t L, double scale) const {
    std::vector<int64_t> coeffs(c_.n, 0);
    const double r = std::nearbyint(value * scale);
    if (!(std::fabs(r) < 4611686018427387904.0)) throw Error("encoded value is too large");
    coeffs[0] = (int64_t)r;
    Plaintext p;
    p.data = DeviceBuffer(c_, (size_t)L * c_.n);
    p.L = L;
    p.scale = scale;
    upload(coeffs.data(), 1, L, p.data.data());
    return p;
}

std::vector<std::vector<cplx>> Encoder::decode_rows(const std::vector<std::vector<double>> &coeffs,
                                                     double scale) const {
    const uint32_t rows = (uint32_t)coeffs.size(), N = c_.n, slots = N / 2;
    shm_context *h = c_.handle();
    std::vector<double> flat((size_t)rows * N, 0.0), re((size_t)rows * slots), im((size_t)rows * slots);
    for (uint32_t r = 0; r < rows; r++)
        for (uint32_t k = 0; k < N && k < coeffs[r].size(); k++) flat[(size_t)r * N + k] = coeffs[r][k];
    DeviceBuffer dc(c_, flat.size()), dre(c_, re.size()), dim(c_, im.size());
    DeviceBuffer ws(c_, shm_encode_workspace_bytes(h, rows) / 8 + 1);
    c_.check(shm_memcpy(h, dc.data(), flat.data(), flat.size() * 8, SHM_COPY_H2D, c_.stream()));
    c_.check(shm_decode(h, reinterpret_cast<const double *>(dc.data()), rows, scale,
                        reinterpret_cast<double *>(dre.data()), reinterpret_cast<double *>(dim.data()), ws.data(),
                        ws.words() * 8, c_.stream()));
    c_.check(shm_memcpy(h, re.data(), dre.data(), re.size() * 8, SHM_COPY_D2H, c_.stream()));
    c_.check(shm_memcpy(h, im.data(), dim.data(), im.size() * 8, SHM_COPY_D2H, c_.stream()));
    std::vector<std::vector<cplx>> out(rows, std::vector<cplx>(slots));
    for (uint32_t r = 0; r < rows; r++)
        for (uint32_t j = 0; j < slots; j++) out[r][j] = cplx(re[(size_t)r * slots + j], im[(size_t)r * slots + j]);
    return out;
}

std::vector<cplx> Encoder::decode(const std::vector<double> &coeffs, double scale) const {
    return decode_rows({coeffs}, scale)[0];
}

// ------------------------------------------------------------------ KeyGenerator

KeyGenerator::KeyGenerator(const Context &c, uint32_t hamming_weight, uint64_t seed)
    : c_(c), enc_(c), seed_(seed) {
    s_coeffs_ = ternary(hamming_weight);
    s_ = ntt_qp(s_coeffs_);
}

void KeyGenerator::import_secrets(const std::vector<int64_t> &s, const std::vector<std::vector<int64_t>> &aux) {
    if (s.size() != c_.n) throw Error("secret has the wrong length");
    for (auto &a : aux)
        if (a.size() != c_.n) throw Error("auxiliary secret has the wrong length");
    DeviceBuffer s_ntt = ntt_qp(s);
    std::vector<DeviceBuffer> aux_ntt;
    for (auto &a : aux) aux_ntt.push_back(ntt_qp(a));
    s_coeffs_ = s;
    s_ = std::move(s_ntt);
    aux_coeffs_ = aux;
    aux_ = std::move(aux_ntt);
}

uint64_t KeyGenerator::next_seed() { return detail::mix64(seed_, ++ctr_); }

// ternary secret with exactly h non-zero coefficients (gen_secretkey and the MOAI
// Hamming-weight trim, secretkey.cu:376-522): partial Fisher-Yates over positions
std::vector<int64_t> KeyGenerator::ternary(uint32_t h) {
    const uint32_t N = c_.n;
    if (h > N) throw Error("Hamming weight above the ring degree");
    const uint64_t sd = next_seed();
    std::vector<uint32_t> idx(N);
    for (uint32_t i = 0; i < N; i++) idx[i] = i;
    std::vector<int64_t> s(N, 0);
    for (uint32_t i = 0; i < h; i++) {
        const uint64_t r = detail::mix64(sd, 2 * (uint64_t)i);
        const uint32_t j = i + (uint32_t)(r % (N - i));
        std::swap(idx[i], idx[j]);
        s[idx[i]] = (detail::mix64(sd, 2 * (uint64_t)i + 1) & 1) ? 1 : -1;
    }
    return s;
}

DeviceBuffer KeyGenerator::ntt_qp(const std::vector<int64_t> &coeffs) const {
    const uint32_t QP = c_.nq + c_.np;
    DeviceBuffer d(c_, (size_t)QP * c_.n);
    enc_.upload(coeffs.data(), 1, QP, d.data());
    return d;
}

std::vector<uint64_t> KeyGenerator::p_units(int digit) const {
    std::vector<uint64_t> unit(c_.nq + c_.np, 0);
    uint32_t lo = 0, hi = c_.nq;
    if (digit >= 0) {
        lo = (uint32_t)digit * c_.np;
        hi = std::min(lo + c_.np, c_.nq);
    }
    for (uint32_t i = lo; i < hi; i++) {
        const uint64_t q = c_.primes[i];
        uint64_t P = 1;
        for (uint32_t k = 0; k < c_.np; k++) P = detail::mulmod(P, c_.primes[c_.nq + k] % q, q);
        unit[i] = P;
    }
    return unit;
}

// [dnum][2][QP][N], digit b = [ e_b - a_b s + P [digit-b CRT unit] s_new , a_b ]
// (generate_one_kswitch_key, secretkey.cu:328-373)
DeviceBuffer KeyGenerator::switching_key(const DeviceBuffer &s_new) {
    std::vector<std::vector<KeyTerm>> adds(c_.dnum);
    for (uint32_t b = 0; b < c_.dnum; b++) adds[b].push_back(KeyTerm{0, p_units((int)b), &s_new});
    return multi_key({&s_}, adds);
}

DeviceBuffer KeyGenerator::multi_key(const std::vector<const DeviceBuffer *> &olds,
                                     const std::vector<std::vector<KeyTerm>> &adds) {
    const uint32_t QP = c_.nq + c_.np, H = (uint32_t)olds.size() + 1;
    const size_t row = (size_t)QP * c_.n;
    DeviceBuffer key(c_, adds.size() * H * row), tmp(c_, row);
    shm_context *h = c_.handle();
    void *st = c_.stream();
    for (size_t d = 0; d < adds.size(); d++) {
        uint64_t *dig = key.data() + d * H * row, *A = dig + (size_t)(H - 1) * row;
        c_.check(shm_sample_uniform(h, A, 1, QP, next_seed(), st));
        for (uint32_t i = 0; i + 1 < H; i++) {
            uint64_t *B = dig + (size_t)i * row;
            c_.check(shm_sample_cbd(h, B, 1, QP, next_seed(), st));
            c_.check(shm_ntt_forward(h, B, 1, QP, st));
            c_.check(shm_multiply_plain(h, A, olds[i]->data(), tmp.data(), 1, QP, st));
            c_.check(shm_sub(h, B, tmp.data(), B, 1, QP, st));
        }
        for (const KeyTerm &t : adds[d]) {
            uint64_t *B = dig + (size_t)t.row * row;
            c_.check(shm_multiply_scalar(h, t.s->data(), t.unit.data(), tmp.data(), 1, QP, st));
            c_.check(shm_add(h, B, tmp.data(), B, 1, QP, st));
        }
    }
    return key;
}

DeviceBuffer KeyGenerator::relin_key() {
    const uint32_t QP = c_.nq + c_.np;
    DeviceBuffer s2(c_, (size_t)QP * c_.n);
    c_.check(shm_multiply_plain(c_.handle(), s_.data(), s_.data(), s2.data(), 1, QP, c_.stream()));
    return switching_key(s2);
}

DeviceBuffer KeyGenerator::public_key() { return multi_key({&s_}, {{}}); }

PublicEncryptor::PublicEncryptor(const Context &c, DeviceBuffer pk, uint64_t seed)
    : c_(c), enc_(c), pk_(std::move(pk)), seed_(seed) {
    if (pk_.words() != 2 * (size_t)(c_.nq + c_.np) * c_.n) throw Error("public key: expected [2][QP][N] words");
}

Ciphertext PublicEncryptor::encrypt_zero(uint32_t count, uint32_t L, double scale) {
    const uint32_t N = c_.n, nq = c_.nq, QP = c_.nq + c_.np;
    if (L < 1 || L > nq) throw Error("level out of range");
    if (!count) throw Error("nothing to encrypt");
    shm_context *h = c_.handle();
    void *st = c_.stream();
    const size_t row = (size_t)QP * N;
    // u: uniform ternary coefficients, one polynomial per ciphertext (sample_ternary_poly)
    std::vector<int64_t> uc((size_t)count * N);
    const uint64_t su = detail::mix64(seed_, ++ctr_);
    for (size_t j = 0; j < uc.size(); j++) uc[j] = (int64_t)(detail::mix64(su, j) % 3) - 1;
    DeviceBuffer u(c_, count * row), x(c_, 2 * count * row), t(c_, row);
    enc_.upload(uc.data(), count, QP, u.data());
    // (e0, e1) over QP, NTT form, then + u * pk
    c_.check(shm_sample_cbd(h, x.data(), 2 * count, QP, detail::mix64(seed_, ++ctr_), st));
    c_.check(shm_ntt_forward(h, x.data(), 2 * count, QP, st));
    for (uint32_t i = 0; i < count; i++)
        for (uint32_t k = 0; k < 2; k++) {
            uint64_t *xi = x.data() + (2 * (size_t)i + k) * row;
            c_.check(shm_multiply_plain(h, u.data() + i * row, pk_.data() + k * row, t.data(), 1, QP, st));
            c_.check(shm_add(h, xi, t.data(), xi, 1, QP, st));
        }
    // ModDown QP -> Q (divide by P), then the first L limbs
    DeviceBuffer q(c_, 2 * (size_t)count * nq * N);
    {
        DeviceBuffer ws(c_, shm_moddown_ext_workspace_bytes(h, 2 * count, nq) / 8 + 1);
        c_.check(shm_moddown_ext(h, x.data(), q.data(), 2 * count, nq, ws.data(), ws.words() * 8, st));
    }
    Ciphertext ct;
    ct.count = count;
    ct.size = 2;
    ct.L = L;
    ct.scale_ = scale;
    if (L == nq) {
        ct.data = std::move(q);
    } else {
        ct.data = DeviceBuffer(c_, 2 * (size_t)count * L * N);
        c_.check(shm_drop_limbs(h, q.data(), ct.data.data(), 2 * count, nq, L, st));
    }
    return ct;
}

Ciphertext PublicEncryptor::encrypt(const std::vector<std::vector<cplx>> &z, double scale, uint32_t L) {
    const uint32_t count = (uint32_t)z.size();
    Ciphertext ct = encrypt_zero(count, L, scale);
    // + the message on c0
    const size_t ln = (size_t)L * c_.n;
    DeviceBuffer m(c_, count * ln);
    {
        DeviceBuffer coeffs(c_, (size_t)count * c_.n);
        enc_.encode_rows(z, scale, coeffs.data());
        enc_.lift(coeffs.data(), count, L, m.data());
    }
    for (uint32_t i = 0; i < count; i++) {
        uint64_t *c0 = ct.data.data() + 2 * i * ln;
        c_.check(shm_add(c_.handle(), c0, m.data() + i * ln, c0, 1, L, c_.stream()));
    }
    return ct;
}

Ciphertext PublicEncryptor::encrypt(const Plaintext &pt) {
    Ciphertext ct = encrypt_zero(1, pt.L, pt.scale);
    c_.check(shm_add(c_.handle(), ct.data.data(), pt.data.data(), ct.data.data(), 1, pt.L, c_.stream()));
    return ct;
}

// s(X^elt) in NTT form, permuted on the device from the NTT form of s (equal to the NTT of the
// permuted coefficients: the automorphism only reorders the evaluation points)
DeviceBuffer KeyGenerator::automorph_ntt(const DeviceBuffer &s_ntt, uint32_t elt) const {
    DeviceBuffer out(c_, (size_t)(c_.nq + c_.np) * c_.n);
    c_.check(shm_permute_galois(c_.handle(), s_ntt.data(), elt, out.data(), c_.nq + c_.np, c_.stream()));
    return out;
}

DeviceBuffer KeyGenerator::galois_key(uint32_t elt) { return switching_key(automorph_ntt(s_, elt)); }

std::map<uint32_t, DeviceBuffer> KeyGenerator::galois_keys(const std::vector<uint32_t> &elts) {
    std::map<uint32_t, DeviceBuffer> out;
    for (uint32_t e : elts) out.emplace(e, galois_key(e));
    return out;
}

void KeyGenerator::gen_aux_secrets(uint32_t members, uint32_t hamming_weight) {
    aux_coeffs_.clear();
    aux_.clear();
    for (uint32_t i = 0; i < members; i++) {
        aux_coeffs_.push_back(ternary(hamming_weight));
        aux_.push_back(ntt_qp(aux_coeffs_.back()));
    }
}

// [dnum][n + 1][QP][N]: B_{d,i} = -A_d s'_i + e + P E_d sigma_g(s'_i), A_d shared by the group
DeviceBuffer KeyGenerator::shared_galois_key(uint32_t elt) {
    if (aux_.empty()) throw Error("no auxiliary secrets: call gen_aux_secrets first");
    std::vector<DeviceBuffer> news;
    for (auto &s : aux_) news.push_back(automorph_ntt(s, elt));
    std::vector<const DeviceBuffer *> olds;
    for (auto &a : aux_) olds.push_back(&a);
    std::vector<std::vector<KeyTerm>> adds(c_.dnum);
    for (uint32_t d = 0; d < c_.dnum; d++)
        for (uint32_t i = 0; i < aux_.size(); i++) adds[d].push_back(KeyTerm{i, p_units((int)d), &news[i]});
    return multi_key(olds, adds);
}

// [n][n + 1][QP][N]: digit j = member j's a; B_fmt[j][i] = -a_fmt[j] s'_i + e + [i == j] P s
DeviceBuffer KeyGenerator::format_key() {
    if (aux_.empty()) throw Error("no auxiliary secrets: call gen_aux_secrets first");
    std::vector<const DeviceBuffer *> olds;
    for (auto &a : aux_) olds.push_back(&a);
    std::vector<std::vector<KeyTerm>> adds(aux_.size());
    for (uint32_t j = 0; j < aux_.size(); j++) adds[j].push_back(KeyTerm{j, p_units(-1), &s_});
    return multi_key(olds, adds);
}

std::vector<DeviceBuffer> KeyGenerator::backward_keys() {
    std::vector<DeviceBuffer> out;
    for (auto &a : aux_) out.push_back(switching_key(a));
    return out;
}

SharedAKeys KeyGenerator::shared_keys(uint32_t members, const std::vector<uint32_t> &elts, uint32_t hamming_weight) {
    gen_aux_secrets(members, hamming_weight);
    SharedAKeys k;
    k.members = members;
    k.format = format_key();
    k.backward = backward_keys();
    for (uint32_t e : elts) k.galois.emplace(e, shared_galois_key(e));
    return k;
}

// c0 = e - a s + m, c1 = a (symmetric; the reference's public-key encryption,
// secretkey.cu:15-217, gives ciphertexts of the same form with a larger fresh error)
Ciphertext KeyGenerator::encrypt(const std::vector<std::vector<cplx>> &z, double scale, uint32_t L) {
    const uint32_t count = (uint32_t)z.size(), N = c_.n;
    if (L < 1 || L > c_.nq) throw Error("level out of range");
    shm_context *h = c_.handle();
    void *st = c_.stream();
    const size_t ln = (size_t)L * N;
    DeviceBuffer m(c_, count * ln), a(c_, count * ln), e(c_, count * ln), t(c_, count * ln);
    {
        DeviceBuffer coeffs(c_, (size_t)count * N);  // every row encoded in one batch on the device
        enc_.encode_rows(z, scale, coeffs.data());
        enc_.lift(coeffs.data(), count, L, m.data());
    }
    c_.check(shm_sample_uniform(h, a.data(), count, L, next_seed(), st));
    c_.check(shm_sample_cbd(h, e.data(), count, L, next_seed(), st));
    c_.check(shm_ntt_forward(h, e.data(), count, L, st));
    c_.check(shm_multiply_plain(h, a.data(), s_.data(), t.data(), count, L, st));
    c_.check(shm_sub(h, e.data(), t.data(), e.data(), count, L, st));
    c_.check(shm_add(h, e.data(), m.data(), e.data(), count, L, st));
    Ciphertext ct;
    ct.data = DeviceBuffer(c_, 2 * count * ln);
    ct.count = count;
    ct.size = 2;
    ct.L = L;
    ct.scale_ = scale;
    for (uint32_t i = 0; i < count; i++) {
        c_.check(shm_memcpy(h, ct.data.data() + 2 * i * ln, e.data() + i * ln, ln * 8, SHM_COPY_D2D, st));
        c_.check(shm_memcpy(h, ct.data.data() + (2 * i + 1) * ln, a.data() + i * ln, ln * 8, SHM_COPY_D2D, st));
    }
    return ct;
}

// m_i = b_i + a s_i on limb 0 (s_i = s for ordinary ciphertexts, s'_i for shared-a
// members), centred; inverse NTT on the device
std::vector<std::vector<double>> KeyGenerator::decrypt_coeffs(const Ciphertext &ct) {
    const uint32_t N = c_.n, mem = ct.members();
    if (ct.size != (ct.shared ? mem + 1 : 2u)) throw Error("decrypt: not a size-2 ciphertext or shared-a group");
    if (ct.shared && mem != aux_.size()) throw Error("decrypt: group size differs from the auxiliary secrets");
    shm_context *h = c_.handle();
    void *st = c_.stream();
    const size_t polys = ct.polys();
    DeviceBuffer l0(c_, polys * N);
    c_.check(shm_drop_limbs(h, ct.data.data(), l0.data(), (uint32_t)polys, ct.L, 1, st));
    std::vector<uint64_t> d(polys * N);
    c_.check(shm_memcpy(h, d.data(), l0.data(), d.size() * 8, SHM_COPY_D2H, st));
    std::vector<std::vector<uint64_t>> sk;
    for (uint32_t i = 0; i < mem; i++) {
        const DeviceBuffer &s = ct.shared ? aux_[i] : s_;
        sk.emplace_back(N);
        c_.check(shm_memcpy(h, sk.back().data(), s.data(), N * 8, SHM_COPY_D2H, st));
    }
    const uint64_t q0 = c_.primes[0];
    const size_t rows = (size_t)ct.count * mem;
    std::vector<uint64_t> m(rows * N);
    for (uint32_t g = 0; g < ct.count; g++)
        for (uint32_t i = 0; i < mem; i++) {
            const uint64_t *b = d.data() + ((size_t)g * ct.size + i) * N;
            const uint64_t *a = d.data() + ((size_t)g * ct.size + ct.size - 1) * N;
            uint64_t *o = m.data() + ((size_t)g * mem + i) * N;
            for (uint32_t k = 0; k < N; k++) o[k] = detail::addmod(b[k], detail::mulmod(a[k], sk[i][k], q0), q0);
        }
    DeviceBuffer md(c_, rows * N);
    c_.check(shm_memcpy(h, md.data(), m.data(), m.size() * 8, SHM_COPY_H2D, st));
    c_.check(shm_ntt_inverse(h, md.data(), (uint32_t)rows, 1, st));
    c_.check(shm_memcpy(h, m.data(), md.data(), m.size() * 8, SHM_COPY_D2H, st));
    std::vector<std::vector<double>> out(rows, std::vector<double>(N));
    for (size_t r = 0; r < rows; r++)
        for (uint32_t k = 0; k < N; k++) {
            const uint64_t v = m[r * N + k];
            out[r][k] = v > q0 / 2 ? -(double)(q0 - v) : (double)v;
        }
    return out;
}

std::vector<std::vector<cplx>> KeyGenerator::decrypt(const Ciphertext &ct) {
    return enc_.decode_rows(decrypt_coeffs(ct), ct.scale_);
}

}  // namespace shmoai
