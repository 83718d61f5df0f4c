// moai::Evaluator over ciphertext batches with exact scale tracking
// (reference: src/include/source/ckks_evaluator_parallel.cuh:150-560 and the Phantom
// free functions of thirdparty/phantom-fhe/include/evaluate.cuh:23-315).  Every
// operation is one C-ABI call for the whole batch.
#include <algorithm>
#include <cmath>

#include "internal.hpp"

namespace shmoai {

Evaluator::Evaluator(const Context &c, const Encoder &enc) : c_(c), enc_(enc) {}

bool Evaluator::same_scale(double a, double b, double rel) {
    return std::fabs(a - b) <= rel * std::max(std::fabs(a), std::fabs(b));
}

uint64_t *Evaluator::ws(size_t bytes) const {
    if (ws_.words() * 8 < bytes) ws_ = DeviceBuffer(c_, (bytes + 7) / 8);
    return ws_.data();
}

void Evaluator::release_workspace() const { ws_ = DeviceBuffer(); }

Ciphertext Evaluator::like(const Ciphertext &a, uint32_t L) const {
    Ciphertext o;
    o.data = DeviceBuffer(c_, a.polys() * L * c_.n);
    o.count = a.count;
    o.size = a.size;
    o.L = L;
    o.scale_ = a.scale_;
    o.shared = a.shared;
    return o;
}

// residues mod q_0 .. q_{L-1} of the integer held exactly by the double v
std::vector<uint64_t> Evaluator::residues(double v, uint32_t L) const {
    std::vector<uint64_t> r(L, 0);
    if (v == 0.0) return r;
    if (!std::isfinite(v) || v != std::nearbyint(v)) throw Error("constant is not an integer: " + std::to_string(v));
    const bool neg = v < 0;
    int e = 0;
    const double m = std::frexp(std::fabs(v), &e);
    uint64_t M = (uint64_t)std::ldexp(m, 53);
    int sh = e - 53;
    if (sh < 0) {
        M >>= -sh;  // exact: the value is an integer
        sh = 0;
    }
    for (uint32_t i = 0; i < L; i++) {
        const uint64_t q = c_.primes[i];
        uint64_t x = detail::mulmod(M % q, detail::powmod(2, (uint64_t)sh, q), q);
        r[i] = (neg && x) ? q - x : x;
    }
    return r;
}

Ciphertext Evaluator::mod_switch_to(const Ciphertext &a, uint32_t L) const {
    if (L > a.L || L < 1) throw Error("cannot raise the level by dropping");
    Ciphertext o = like(a, L);
    c_.check(shm_drop_limbs(c_.handle(), a.data.data(), o.data.data(), (uint32_t)a.polys(), a.L, L, c_.stream()));
    return o;
}

static void same_shape(const Ciphertext &a, const Ciphertext &b) {
    if (a.count != b.count || a.size != b.size || a.shared != b.shared)
        throw Error("ciphertext batches of different shapes");
}

Ciphertext Evaluator::add(const Ciphertext &a, const Ciphertext &b) const {
    if (a.size != b.size && !a.shared && !b.shared && a.count == b.count) {
        // an unrelinearised product plus an ordinary ciphertext (evaluate.cu:114-160 extends
        // the shorter operand with zero polynomials)
        if (!same_scale(a.scale_, b.scale_)) throw Error("scale mismatch in add");
        if (a.L != b.L) {
            const uint32_t L = std::min(a.L, b.L);
            return a.L > L ? add(mod_switch_to(a, L), b) : add(a, mod_switch_to(b, L));
        }
        const Ciphertext &big = a.size > b.size ? a : b, &small = a.size > b.size ? b : a;
        Ciphertext o = like(big, big.L);
        c_.check(shm_add_sizes(c_.handle(), big.data.data(), big.size, small.data.data(), small.size, o.data.data(),
                               a.count, a.L, c_.stream()));
        return o;
    }
    same_shape(a, b);
    if (!same_scale(a.scale_, b.scale_)) throw Error("scale mismatch in add");
    if (a.L != b.L) {
        const uint32_t L = std::min(a.L, b.L);
        return a.L > L ? add(mod_switch_to(a, L), b) : add(a, mod_switch_to(b, L));
    }
    Ciphertext o = like(a, a.L);
    c_.check(shm_add(c_.handle(), a.data.data(), b.data.data(), o.data.data(), (uint32_t)a.polys(), a.L,
                     c_.stream()));
    return o;
}

Ciphertext Evaluator::sub(const Ciphertext &a, const Ciphertext &b) const {
    same_shape(a, b);
    if (!same_scale(a.scale_, b.scale_)) throw Error("scale mismatch in sub");
    if (a.L != b.L) {
        const uint32_t L = std::min(a.L, b.L);
        return a.L > L ? sub(mod_switch_to(a, L), b) : sub(a, mod_switch_to(b, L));
    }
    Ciphertext o = like(a, a.L);
    c_.check(shm_sub(c_.handle(), a.data.data(), b.data.data(), o.data.data(), (uint32_t)a.polys(), a.L,
                     c_.stream()));
    return o;
}

Ciphertext Evaluator::negate(const Ciphertext &a) const {
    Ciphertext o = like(a, a.L);
    c_.check(shm_negate(c_.handle(), a.data.data(), o.data.data(), (uint32_t)a.polys(), a.L, c_.stream()));
    return o;
}

Ciphertext Evaluator::multiply_plain(const Ciphertext &a, const Plaintext &p) const {
    if (p.L < a.L) throw Error("plaintext has fewer limbs than the ciphertext");
    Ciphertext o = like(a, a.L);
    c_.check(shm_multiply_plain(c_.handle(), a.data.data(), p.data.data(), o.data.data(), (uint32_t)a.polys(), a.L,
                                c_.stream()));
    o.scale_ = a.scale_ * p.scale;
    return o;
}

Ciphertext Evaluator::multiply_int(const Ciphertext &a, int64_t k) const {
    std::vector<uint64_t> r(a.L);
    for (uint32_t i = 0; i < a.L; i++) {
        const uint64_t q = c_.primes[i];
        const int64_t m = k % (int64_t)q;
        r[i] = m < 0 ? (uint64_t)(m + (int64_t)q) : (uint64_t)m;
    }
    Ciphertext o = like(a, a.L);
    c_.check(shm_multiply_scalar(c_.handle(), a.data.data(), r.data(), o.data.data(), (uint32_t)a.polys(), a.L,
                                 c_.stream()));
    return o;
}

Ciphertext Evaluator::add_const(const Ciphertext &a, double c) const {
    if (a.shared || a.size != 2) throw Error("add_const needs ordinary size-2 ciphertexts");
    std::vector<uint64_t> r = residues(std::nearbyint(c * a.scale_), a.L);
    Ciphertext o = like(a, a.L);
    c_.check(shm_add_scalar(c_.handle(), a.data.data(), r.data(), o.data.data(), a.count, a.L, c_.stream()));
    return o;
}

Ciphertext Evaluator::rescale_to_next(const Ciphertext &a) const {
    if (a.L < 2) throw Error("no prime left to rescale by");
    Ciphertext o = like(a, a.L - 1);
    const uint32_t p = (uint32_t)a.polys();
    uint64_t *w = ws(shm_rescale_workspace_bytes(c_.handle(), p, a.L));
    c_.check(shm_rescale(c_.handle(), a.data.data(), o.data.data(), p, a.L, w, ws_.words() * 8, c_.stream()));
    o.scale_ = a.scale_ / (double)c_.primes[a.L - 1];
    return o;
}

Ciphertext Evaluator::multiply_const(const Ciphertext &a, double c, double target) const {
    const double q = (double)c_.primes[a.L - 1];
    const double T = target * q / a.scale_;
    std::vector<uint64_t> r = residues(std::nearbyint(c * T), a.L);
    Ciphertext t = like(a, a.L);
    c_.check(shm_multiply_scalar(c_.handle(), a.data.data(), r.data(), t.data.data(), (uint32_t)a.polys(), a.L,
                                 c_.stream()));
    Ciphertext o = rescale_to_next(t);
    o.scale_ = target;
    return o;
}

Ciphertext Evaluator::linear_combination(const std::vector<const Ciphertext *> &X, const std::vector<double> &w,
                                         double w0, uint32_t L, double scale) const {
    if (X.empty() || X.size() != w.size() || X.size() > 8) throw Error("linear_combination: 1..8 terms and weights");
    std::vector<const uint64_t *> xp;
    std::vector<uint32_t> lv;
    std::vector<uint64_t> wr;
    for (size_t i = 0; i < X.size(); i++) {
        const Ciphertext &x = *X[i];
        if (x.shared || x.size != 2 || x.count != X[0]->count) throw Error("linear_combination: size-2 batches of one count");
        if (x.L < L) throw Error("linear_combination: a term has fewer primes than the result");
        xp.push_back(x.data.data());
        lv.push_back(x.L);
        const std::vector<uint64_t> r = residues(w[i], L);
        wr.insert(wr.end(), r.begin(), r.end());
    }
    const std::vector<uint64_t> r0 = residues(w0, L);
    Ciphertext o;
    o.data = DeviceBuffer(c_, (size_t)X[0]->count * 2 * L * c_.n);
    o.count = X[0]->count;
    o.L = L;
    o.scale_ = scale;
    c_.check(shm_linear_combination(c_.handle(), xp.data(), lv.data(), wr.data(), (uint32_t)xp.size(),
                                    w0 != 0.0 ? r0.data() : nullptr, o.data.data(), o.count, L, c_.stream()));
    return o;
}

Ciphertext Evaluator::multiply_const_unscaled(const Ciphertext &a, double c, double T) const {
    std::vector<uint64_t> r = residues(std::nearbyint(c * T), a.L);
    Ciphertext o = like(a, a.L);
    c_.check(shm_multiply_scalar(c_.handle(), a.data.data(), r.data(), o.data.data(), (uint32_t)a.polys(), a.L,
                                 c_.stream()));
    o.scale_ = a.scale_ * T;
    return o;
}

// bring a to (L, scale): a pure drop when the scale already matches, otherwise a drop
// to L + 1 and one exact constant multiply
Ciphertext Evaluator::adjust(const Ciphertext &a, uint32_t L, double scale) const {
    if (a.L <= L) {
        if (!same_scale(a.scale_, scale)) throw Error("cannot adjust the scale without a spare level");
        Ciphertext o = like(a, a.L);
        c_.check(shm_memcpy(c_.handle(), o.data.data(), a.data.data(), a.polys() * a.L * c_.n * 8, SHM_COPY_D2D,
                            c_.stream()));
        o.scale_ = scale;
        return o;
    }
    if (same_scale(a.scale_, scale)) {
        Ciphertext o = mod_switch_to(a, L);
        o.scale_ = scale;
        return o;
    }
    if (a.L > L + 1) return multiply_const(mod_switch_to(a, L + 1), 1.0, scale);
    return multiply_const(a, 1.0, scale);
}

Ciphertext Evaluator::multiply_lazy(const Ciphertext &a, const Ciphertext &b) const {
    if (a.shared || b.shared || a.size != 2 || b.size != 2) throw Error("multiply needs ordinary ciphertexts");
    if (a.count != b.count) throw Error("batches of different sizes");
    if (a.L != b.L) {
        const uint32_t L = std::min(a.L, b.L);
        return a.L > L ? multiply_lazy(mod_switch_to(a, L), b) : multiply_lazy(a, mod_switch_to(b, L));
    }
    Ciphertext r;
    r.data = DeviceBuffer(c_, (size_t)a.count * 3 * a.L * c_.n);
    r.count = a.count;
    r.size = 3;
    r.L = a.L;
    r.scale_ = a.scale_ * b.scale_;
    c_.check(shm_multiply(c_.handle(), a.data.data(), b.data.data(), r.data.data(), a.count, a.L, c_.stream()));
    return r;
}

Ciphertext Evaluator::multiply_accumulate(const std::vector<const Ciphertext *> &A,
                                          const std::vector<const Ciphertext *> &B) const {
    if (A.empty() || A.size() != B.size()) throw Error("multiply_accumulate: bad term lists");
    const uint32_t count = A[0]->count;
    uint32_t L = A[0]->L;
    const bool bcast = B[0]->count == 1 && count > 1;
    for (size_t t = 0; t < A.size(); t++) {
        const Ciphertext &a = *A[t], &b = *B[t];
        if (a.shared || b.shared || a.size != 2 || b.size != 2) throw Error("multiply needs ordinary ciphertexts");
        if (a.count != count || b.count != (bcast ? 1 : count)) throw Error("multiply_accumulate: batch sizes differ");
        if (!same_scale(a.scale_ * b.scale_, A[0]->scale_ * B[0]->scale_)) throw Error("scale mismatch in add");
        L = std::min(L, std::min(a.L, b.L));
    }
    // terms above the common level are dropped to it (kept alive here for the call)
    std::vector<Ciphertext> dropped;
    dropped.reserve(2 * A.size());
    std::vector<const uint64_t *> pa(A.size()), pb(B.size());
    for (size_t t = 0; t < A.size(); t++) {
        const Ciphertext *a = A[t], *b = B[t];
        if (a->L != L) {
            dropped.push_back(mod_switch_to(*a, L));
            a = &dropped.back();
        }
        if (b->L != L) {
            dropped.push_back(mod_switch_to(*b, L));
            b = &dropped.back();
        }
        pa[t] = a->data.data();
        pb[t] = b->data.data();
    }
    Ciphertext r;
    r.data = DeviceBuffer(c_, (size_t)count * 3 * L * c_.n);
    r.count = count;
    r.size = 3;
    r.L = L;
    r.scale_ = A[0]->scale_ * B[0]->scale_;
    c_.check(shm_multiply_accumulate(c_.handle(), pa.data(), pb.data(), (uint32_t)A.size(), bcast ? 1 : 0,
                                     r.data.data(), count, L, 0, c_.stream()));
    return r;
}

Ciphertext Evaluator::sum_of_products(const Ciphertext &X, const Ciphertext &W) const {
    if (X.shared || W.shared || X.size != 2 || W.size != 2) throw Error("multiply needs ordinary ciphertexts");
    if (X.count != W.count || X.count == 0) throw Error("sum_of_products: batches of different sizes");
    if (X.L != W.L) {
        const uint32_t L = std::min(X.L, W.L);
        return X.L > L ? sum_of_products(mod_switch_to(X, L), W) : sum_of_products(X, mod_switch_to(W, L));
    }
    const size_t per = (size_t)2 * X.L * c_.n;
    std::vector<const uint64_t *> pa(X.count), pb(X.count);
    for (uint32_t j = 0; j < X.count; j++) {
        pa[j] = X.data.data() + j * per;
        pb[j] = W.data.data() + j * per;
    }
    Ciphertext r;
    r.data = DeviceBuffer(c_, (size_t)3 * X.L * c_.n);
    r.count = 1;
    r.size = 3;
    r.L = X.L;
    r.scale_ = X.scale_ * W.scale_;
    c_.check(shm_multiply_accumulate(c_.handle(), pa.data(), pb.data(), X.count, 0, r.data.data(), 1, X.L, 0,
                                     c_.stream()));
    return r;
}

Ciphertext Evaluator::relinearize(const Ciphertext &a) const {
    if (a.shared || a.size != 3) throw Error("relinearize takes size-3 ciphertexts");
    if (!relin_key) throw Error("no relinearisation key");
    Ciphertext r;
    r.data = DeviceBuffer(c_, (size_t)a.count * 2 * a.L * c_.n);
    r.count = a.count;
    r.L = a.L;
    r.scale_ = a.scale_;
    uint64_t *w = ws(shm_keyswitch_workspace_bytes(c_.handle(), a.count, a.L));
    c_.check(shm_relinearize(c_.handle(), a.data.data(), relin_key->data(), r.data.data(), a.count, a.L, w,
                             ws_.words() * 8, c_.stream()));
    return r;
}

Ciphertext Evaluator::relinearize_rescale(const Ciphertext &a) const {
    if (a.shared || a.size != 3) throw Error("relinearize_rescale takes size-3 ciphertexts");
    if (!relin_key) throw Error("no relinearisation key");
    if (a.L < 2) throw Error("no prime left to rescale by");
    Ciphertext r;
    r.data = DeviceBuffer(c_, (size_t)a.count * 2 * (a.L - 1) * c_.n);
    r.count = a.count;
    r.L = a.L - 1;
    r.scale_ = a.scale_ / (double)c_.primes[a.L - 1];
    uint64_t *w = ws(shm_keyswitch_workspace_bytes(c_.handle(), a.count, a.L));
    c_.check(shm_relinearize_rescale(c_.handle(), a.data.data(), relin_key->data(), r.data.data(), a.count, a.L, w,
                                     ws_.words() * 8, c_.stream()));
    return r;
}

Ciphertext Evaluator::multiply(const Ciphertext &a, const Ciphertext &b, bool rescale) const {
    if (a.shared || b.shared || a.size != 2 || b.size != 2) throw Error("multiply needs ordinary ciphertexts");
    if (a.count != b.count) throw Error("batches of different sizes");
    if (!relin_key) throw Error("no relinearisation key");
    if (a.L != b.L) {
        const uint32_t L = std::min(a.L, b.L);
        return a.L > L ? multiply(mod_switch_to(a, L), b, rescale) : multiply(a, mod_switch_to(b, L), rescale);
    }
    const size_t ln = (size_t)a.L * c_.n;
    DeviceBuffer t3(c_, (size_t)a.count * 3 * ln);
    c_.check(shm_multiply(c_.handle(), a.data.data(), b.data.data(), t3.data(), a.count, a.L, c_.stream()));
    Ciphertext r = like(a, a.L);
    uint64_t *w = ws(shm_keyswitch_workspace_bytes(c_.handle(), a.count, a.L));
    c_.check(shm_relinearize(c_.handle(), t3.data(), relin_key->data(), r.data.data(), a.count, a.L, w,
                             ws_.words() * 8, c_.stream()));
    r.scale_ = a.scale_ * b.scale_;
    if (rescale) return rescale_to_next(r);
    return r;
}

Ciphertext Evaluator::multiply_plain_accumulate(const std::vector<const Ciphertext *> &X,
                                                const std::vector<const Plaintext *> &P) const {
    if (X.empty() || X.size() != P.size()) throw Error("multiply_plain_accumulate: bad term lists");
    const Ciphertext &x0 = *X[0];
    std::vector<const uint64_t *> xp, pp;
    for (size_t i = 0; i < X.size(); i++) {
        if (X[i]->L != x0.L || X[i]->count != x0.count || X[i]->size != x0.size)
            throw Error("multiply_plain_accumulate: terms of different shapes");
        if (P[i]->L < x0.L) throw Error("plaintext has fewer limbs than the ciphertext");
        xp.push_back(X[i]->data.data());
        pp.push_back(P[i]->data.data());
    }
    Ciphertext o = like(x0, x0.L);
    c_.check(shm_multiply_plain_accumulate(c_.handle(), xp.data(), pp.data(), (uint32_t)xp.size(), o.data.data(),
                                           (uint32_t)x0.polys(), x0.L, 0, c_.stream()));
    o.scale_ = x0.scale_ * P[0]->scale;
    return o;
}

uint32_t Evaluator::galois_elt(int step) const {
    const uint64_t n2 = 2ull * c_.n, slots = c_.n / 2;
    if (step == 0) return (uint32_t)(n2 - 1);
    const int64_t s = ((int64_t)step % (int64_t)slots + (int64_t)slots) % (int64_t)slots;
    return (uint32_t)detail::powmod(5, (uint64_t)s, n2);
}

// automorphisms of one batch by several elements with one hoisted ModUp (Sh-Rot for shared-a)
std::vector<Ciphertext> Evaluator::automorphisms(const Ciphertext &a, const std::vector<uint32_t> &elts) const {
    const std::map<uint32_t, DeviceBuffer> *table = nullptr;
    if (a.shared) {
        if (!shared_keys || shared_keys->members != a.members())
            throw Error("no shared-a keys for this group size");
        table = &shared_keys->galois;
    } else {
        if (a.size != 2) throw Error("rotation needs size-2 ciphertexts");
        if (!galois_keys) throw Error("no Galois keys");
        table = galois_keys;
    }
    std::vector<const uint64_t *> keys;
    std::vector<Ciphertext> outs;
    std::vector<uint64_t *> optr;
    for (uint32_t e : elts) {
        auto it = table->find(e);
        if (it == table->end()) throw Error("missing Galois key for element " + std::to_string(e));
        keys.push_back(it->second.data());
        outs.push_back(like(a, a.L));
        optr.push_back(outs.back().data.data());
    }
    shm_context *h = c_.handle();
    const uint32_t k = (uint32_t)elts.size();
    if (a.shared) {
        uint64_t *w = ws(shm_shared_rotate_workspace_bytes(h, a.count, a.members(), a.L));
        c_.check(shm_shared_rotate_hoisted(h, a.data.data(), a.count, a.members(), k, elts.data(), keys.data(),
                                           optr.data(), a.L, w, ws_.words() * 8, c_.stream()));
    } else if (k == 1) {
        uint64_t *w = ws(shm_keyswitch_workspace_bytes(h, a.count, a.L) + (size_t)a.count * 2 * a.L * c_.n * 8);
        c_.check(shm_apply_galois(h, a.data.data(), elts[0], keys[0], optr[0], a.count, a.L, w, ws_.words() * 8,
                                  c_.stream()));
    } else {
        uint64_t *w = ws(shm_apply_galois_hoisted_workspace_bytes(h, a.count, a.L));
        c_.check(shm_apply_galois_hoisted(h, a.data.data(), k, elts.data(), keys.data(), optr.data(), a.count, a.L, w,
                                          ws_.words() * 8, c_.stream()));
    }
    return outs;
}

Ciphertext Evaluator::rotate_vector(const Ciphertext &a, int step) const {
    if (step % (int)(c_.n / 2) == 0) {
        Ciphertext o = like(a, a.L);
        c_.check(shm_memcpy(c_.handle(), o.data.data(), a.data.data(), a.polys() * a.L * c_.n * 8, SHM_COPY_D2D,
                            c_.stream()));
        return o;
    }
    return std::move(automorphisms(a, {galois_elt(step)})[0]);
}

std::map<int, Ciphertext> Evaluator::rotate_many(const Ciphertext &a, const std::vector<int> &steps) const {
    std::vector<int> st;
    std::vector<uint32_t> elts;
    for (int s : steps)
        if (s % (int)(c_.n / 2)) {
            st.push_back(s);
            elts.push_back(galois_elt(s));
        }
    std::map<int, Ciphertext> out;
    if (st.empty()) return out;
    std::vector<Ciphertext> r = automorphisms(a, elts);
    for (size_t i = 0; i < st.size(); i++) out.emplace(st[i], std::move(r[i]));
    return out;
}

Ciphertext Evaluator::complex_conjugate(const Ciphertext &a) const {
    return std::move(automorphisms(a, {2 * c_.n - 1})[0]);
}

// X^(N/2) in NTT form over the chain primes: multiplying by it multiplies every slot by
// i (omega_j^(N/2) = i for all j), exactly and without a level
const Plaintext &Evaluator::monomial_half() const {
    if (!mono_.L) {
        std::vector<int64_t> c(c_.n, 0);
        c[c_.n / 2] = 1;
        mono_.data = DeviceBuffer(c_, (size_t)c_.nq * c_.n);
        mono_.L = c_.nq;
        mono_.scale = 1.0;
        enc_.upload(c.data(), 1, c_.nq, mono_.data.data());
    }
    return mono_;
}

Ciphertext Evaluator::multiply_i(const Ciphertext &a, int sign) const {
    Ciphertext o = like(a, a.L);
    c_.check(shm_multiply_plain(c_.handle(), a.data.data(), monomial_half().data.data(), o.data.data(),
                                (uint32_t)a.polys(), a.L, c_.stream()));
    if (sign < 0) c_.check(shm_negate(c_.handle(), o.data.data(), o.data.data(), (uint32_t)a.polys(), a.L, c_.stream()));
    return o;
}

Ciphertext Evaluator::mod_raise(const Ciphertext &a, uint32_t L) const {
    if (a.L != 1) throw Error("mod_raise takes one-prime ciphertexts");
    Ciphertext o = like(a, L);
    const uint32_t p = (uint32_t)a.polys();
    uint64_t *w = ws(shm_modraise_workspace_bytes(c_.handle(), p));
    c_.check(shm_modraise(c_.handle(), a.data.data(), o.data.data(), p, L, w, ws_.words() * 8, c_.stream()));
    return o;
}

Ciphertext Evaluator::concat(const Ciphertext &a, const Ciphertext &b) const {
    if (a.L != b.L || a.size != b.size || a.shared != b.shared || !same_scale(a.scale_, b.scale_))
        throw Error("concat: batches differ in level, size or scale");
    Ciphertext o;
    const size_t wa = a.polys() * a.L * c_.n, wb = b.polys() * b.L * c_.n;
    o.data = DeviceBuffer(c_, wa + wb);
    o.count = a.count + b.count;
    o.size = a.size;
    o.L = a.L;
    o.scale_ = a.scale_;
    o.shared = a.shared;
    c_.check(shm_memcpy(c_.handle(), o.data.data(), a.data.data(), wa * 8, SHM_COPY_D2D, c_.stream()));
    c_.check(shm_memcpy(c_.handle(), o.data.data() + wa, b.data.data(), wb * 8, SHM_COPY_D2D, c_.stream()));
    return o;
}

Ciphertext Evaluator::slice(const Ciphertext &a, uint32_t first, uint32_t count) const {
    if (first + count > a.count) throw Error("slice out of range");
    Ciphertext o;
    const size_t per = (size_t)a.size * a.L * c_.n;
    o.data = DeviceBuffer(c_, count * per);
    o.count = count;
    o.size = a.size;
    o.L = a.L;
    o.scale_ = a.scale_;
    o.shared = a.shared;
    c_.check(shm_memcpy(c_.handle(), o.data.data(), a.data.data() + first * per, count * per * 8, SHM_COPY_D2D,
                        c_.stream()));
    return o;
}

Ciphertext Evaluator::ctpt_matmul(const Ciphertext &X, const std::vector<int64_t> &W, uint32_t n_out,
                                  double w_scale, bool tensor_cores) const {
    if (X.shared || X.size != 2) throw Error("ct-pt matmul takes ordinary ciphertexts");
    const uint32_t n_in = X.count;
    if (W.size() != (size_t)n_in * n_out) throw Error("weight matrix must be [n_in][n_out]");
    shm_context *h = c_.handle();
    DeviceBuffer Wd(c_, W.size());
    c_.check(shm_memcpy(h, Wd.data(), W.data(), W.size() * 8, SHM_COPY_H2D, c_.stream()));
    Ciphertext Y;
    Y.data = DeviceBuffer(c_, (size_t)n_out * 2 * X.L * c_.n);
    Y.count = n_out;
    Y.size = 2;
    Y.L = X.L;
    Y.scale_ = X.scale_ * w_scale;
    const int64_t *w = reinterpret_cast<const int64_t *>(Wd.data());
    if (tensor_cores) {
        uint64_t *wsp = ws(shm_ctpt_matmul_workspace_bytes(h, n_in, n_out, X.L));
        c_.check(shm_ctpt_matmul(h, X.data.data(), w, Y.data.data(), n_in, n_out, X.L, wsp, ws_.words() * 8,
                                 c_.stream()));
    } else {
        c_.check(shm_ctpt_matmul_cuda_core(h, X.data.data(), w, Y.data.data(), n_in, n_out, X.L, c_.stream()));
    }
    return rescale_to_next(Y);
}

Ciphertext Evaluator::ctpt_matmul_masked(const Ciphertext &X, const std::vector<int64_t> &W, uint32_t n_out,
                                         double w_scale, const std::vector<double> &mask, bool tensor_cores) const {
    if (mask.size() != c_.n / 2) throw Error("mask needs one value per slot");
    if (X.L < 3) throw Error("masked ct-pt matmul needs two levels and one prime for its output");
    Ciphertext Z = ctpt_matmul(X, W, n_out, w_scale, tensor_cores);
    const std::vector<cplx> m(mask.begin(), mask.end());
    const Plaintext M = enc_.encode(m, Z.L, (double)c_.primes[Z.L - 1]);
    return rescale_to_next(multiply_plain(Z, M));
}

Ciphertext Evaluator::to_shared(const Ciphertext &a, uint32_t members) const {
    if (a.shared || a.size != 2) throw Error("to_shared takes ordinary ciphertexts");
    if (!members || a.count % members) throw Error("batch is not a multiple of the group size");
    if (!shared_keys || shared_keys->members != members || !shared_keys->format.data())
        throw Error("no format key for this group size");
    Ciphertext o;
    const uint32_t G = a.count / members;
    o.data = DeviceBuffer(c_, (size_t)G * (members + 1) * a.L * c_.n);
    o.count = G;
    o.size = members + 1;
    o.L = a.L;
    o.scale_ = a.scale_;
    o.shared = true;
    uint64_t *w = ws(shm_fmt_switch_forward_workspace_bytes(c_.handle(), G, members, a.L));
    c_.check(shm_fmt_switch_forward(c_.handle(), a.data.data(), G, members, shared_keys->format.data(),
                                    o.data.data(), a.L, w, ws_.words() * 8, c_.stream()));
    return o;
}

Ciphertext Evaluator::from_shared(const Ciphertext &a) const {
    if (!a.shared) throw Error("from_shared takes shared-a groups");
    const uint32_t n = a.members();
    if (!shared_keys || shared_keys->members != n || shared_keys->backward.size() != n)
        throw Error("no backward keys for this group size");
    std::vector<const uint64_t *> keys;
    for (auto &k : shared_keys->backward) keys.push_back(k.data());
    Ciphertext o;
    o.data = DeviceBuffer(c_, (size_t)a.count * n * 2 * a.L * c_.n);
    o.count = a.count * n;
    o.size = 2;
    o.L = a.L;
    o.scale_ = a.scale_;
    o.shared = false;
    uint64_t *w = ws(shm_fmt_switch_backward_workspace_bytes(c_.handle(), a.count, n, a.L));
    c_.check(shm_fmt_switch_backward(c_.handle(), a.data.data(), a.count, n, keys.data(), o.data.data(), a.L, w,
                                     ws_.words() * 8, c_.stream()));
    return o;
}

}  // namespace shmoai
