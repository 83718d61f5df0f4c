// The softmax's and LayerNorm's building blocks on ciphertext batches (src/include/source/
// non_linear_func/softmax.cuh:23-118, layernorm.cuh:708-897): exp by (1 + x/128)^128, 1/x by
// the product prod_i (1 + y^(2^i)), y = 1 - x, and 1/sqrt(x) by Newton and Goldschmidt steps.
// Products are relinearised and rescaled in one ModDown (relinearize_rescale).
#include <algorithm>
#include <cmath>

#include "internal.hpp"

namespace shmoai {

namespace {

Ciphertext square(const Evaluator &ev, const Ciphertext &a) { return ev.relinearize_rescale(ev.multiply_lazy(a, a)); }

Ciphertext product(const Evaluator &ev, const Ciphertext &a, const Ciphertext &b) {
    return ev.relinearize_rescale(ev.multiply_lazy(a, b));
}

void need_ordinary(const Ciphertext &x, const char *what) {
    if (x.shared || x.size != 2) throw Error(std::string(what) + " takes ordinary size-2 ciphertexts");
}

}  // namespace

// exp (softmax.cuh:23-76): u = x / 128 + 1 (one scalar product, its output scale set to the
// prime the first square divides by), then seven squarings: 8 levels
Ciphertext exp_approx(const Evaluator &ev, const Ciphertext &x) {
    need_ordinary(x, "exp");
    if (x.L < 9) throw Error("exp needs 8 levels and one prime for its output");
    const Context &c = ev.context();
    Ciphertext y = ev.add_const(ev.multiply_const(x, 1.0 / 128.0, (double)c.primes[x.L - 2]), 1.0);
    for (int i = 0; i < 7; i++) y = square(ev, y);
    return y;
}

// 1/x for x in (0, 2) (softmax.cuh:78-118): y = 1 - x, r = 1 + y, then per iteration
// y <- y^2 and r <- r (1 + y), so r = prod_{i <= iter} (1 + y^(2^i)) = (1 - y^(2^(iter+1))) / x;
// iter levels plus one for the alignment of the first product
Ciphertext inverse_approx(const Evaluator &ev, const Ciphertext &x, int iter) {
    need_ordinary(x, "inverse");
    if (iter < 1) throw Error("inverse needs at least one iteration");
    if ((int)x.L < iter + 2) throw Error("inverse needs iter + 1 levels and one prime for its output");
    Ciphertext y = ev.add_const(ev.multiply_int(x, -1), 1.0);
    Ciphertext r = ev.add_const(y, 1.0);
    for (int i = 0; i < iter; i++) {
        y = square(ev, y);
        r = product(ev, r, ev.add_const(y, 1.0));
    }
    return r;
}

// a + b after bringing both to the lower level and b to a's scale (b is scaled by one exact
// constant multiply when the scales differ, which needs a spare level on b)
static Ciphertext add_aligned(const Evaluator &ev, const Ciphertext &a, const Ciphertext &b) {
    const uint32_t L = std::min(a.L, b.L);
    const bool same = std::fabs(a.scale_ / b.scale_ - 1.0) < 1e-12;
    if (same) return ev.add(ev.mod_switch_to(a, L), ev.mod_switch_to(b, L));
    // the rescaled copy of b lands one level lower: bring a there too
    const uint32_t Lb = std::min(L + 1, b.L);
    Ciphertext bs = ev.multiply_const(ev.mod_switch_to(b, Lb), 1.0, a.scale_);
    const uint32_t Lo = std::min(bs.L, L);
    Ciphertext ao = ev.mod_switch_to(a, Lo);
    return ev.add(ao, ev.mod_switch_to(bs, Lo));
}

// 1/sqrt(x) (invert_sqrt, layernorm.cuh:708-897): the line -1.29054537e-4 x + 0.129054537 as
// the first guess, d_newt Newton steps r <- r (3/2 - x r^2 / 2), then d_gold Goldschmidt steps
// on (g, h) = (x r, r / 2): s = 1/2 - g h, g <- g + g s, h <- h + h s; the result is 2 h
Ciphertext inv_sqrt_approx(const Evaluator &ev, const Ciphertext &x, int d_newt, int d_gold) {
    need_ordinary(x, "inverse square root");
    if (d_newt < 0 || d_gold < 0) throw Error("iteration counts must be non-negative");
    const uint32_t need = 2 * (uint32_t)(d_newt + d_gold) + 4;  // levels used + the output prime
    if (x.L < need) throw Error("inverse square root needs " + std::to_string(need) + " primes");
    const Context &c = ev.context();
    const double S = x.scale_;
    Ciphertext r = ev.add_const(ev.multiply_const(x, -1.29054537e-4, (double)c.primes[x.L - 2]), 1.29054537e-1);
    const Ciphertext xh = ev.multiply_const(x, -0.5, (double)c.primes[x.L - 2]);  // -x / 2
    for (int i = 0; i < d_newt; i++) {
        Ciphertext t = product(ev, product(ev, xh, r), square(ev, r));  // -x r^3 / 2
        r = add_aligned(ev, t, ev.multiply_const(r, 1.5, (double)c.primes[r.L - 2]));
    }
    Ciphertext g = product(ev, x, r);
    Ciphertext h = ev.multiply_const(r, 0.5, (double)c.primes[r.L - 2]);
    for (int i = 0; i < d_gold; i++) {
        Ciphertext s = ev.add_const(ev.multiply_int(product(ev, g, h), -1), 0.5);
        Ciphertext g2 = product(ev, g, s), h2 = product(ev, h, s);
        g = add_aligned(ev, g2, g);
        h = add_aligned(ev, h2, h);
    }
    Ciphertext out = ev.multiply_const(h, 2.0, S);
    return out;
}

Ciphertext batch_sum(const Evaluator &ev, const Ciphertext &x) {
    need_ordinary(x, "batch_sum");
    if (x.count == 0) throw Error("empty batch");
    Ciphertext cur = ev.slice(x, 0, x.count);
    while (cur.count > 1) {  // halves added pairwise; an odd last member is carried
        const uint32_t h = cur.count / 2;
        Ciphertext s = ev.add(ev.slice(cur, 0, h), ev.slice(cur, h, h));
        if (cur.count & 1) s = ev.concat(s, ev.slice(cur, 2 * h, 1));
        cur = std::move(s);
    }
    return cur;
}

static Ciphertext gather_ptrs(const Evaluator &ev, const std::vector<const Ciphertext *> &parts) {
    if (parts.empty()) throw Error("nothing to gather");
    const Ciphertext &p0 = *parts[0];
    const Context &c = ev.context();
    size_t words = 0;
    uint32_t count = 0;
    for (const Ciphertext *p : parts) {
        if (p->L != p0.L || p->size != p0.size || p->shared != p0.shared ||
            std::fabs(p->scale_ / p0.scale_ - 1.0) > 1e-12)
            throw Error("gather: parts differ in level, size or scale");
        words += p->polys() * p->L * c.n;
        count += p->count;
    }
    Ciphertext o;
    o.data = DeviceBuffer(c, words);
    o.count = count;
    o.size = p0.size;
    o.L = p0.L;
    o.scale_ = p0.scale_;
    o.shared = p0.shared;
    size_t off = 0;
    for (const Ciphertext *p : parts) {
        const size_t w = p->polys() * p->L * c.n;
        c.check(shm_memcpy(c.handle(), o.data.data() + off, p->data.data(), w * 8, SHM_COPY_D2D, c.stream()));
        off += w;
    }
    return o;
}

Ciphertext batch_broadcast(const Evaluator &ev, const Ciphertext &one, uint32_t count) {
    if (count == 0) throw Error("broadcast to an empty batch");
    return gather_ptrs(ev, std::vector<const Ciphertext *>(count, &one));
}

Ciphertext batch_gather(const Evaluator &ev, const std::vector<Ciphertext> &parts) {
    std::vector<const Ciphertext *> p;
    for (const Ciphertext &x : parts) p.push_back(&x);
    return gather_ptrs(ev, p);
}

// each part is released (stream-ordered, after its copy) as soon as it is copied, so the gathered
// batch and the parts together never take much more than one batch of device memory
Ciphertext batch_gather(const Evaluator &ev, std::vector<Ciphertext> &&parts) {
    if (parts.size() == 1) {
        Ciphertext o = std::move(parts[0]);
        parts.clear();
        return o;
    }
    Ciphertext o;
    {
        std::vector<const Ciphertext *> p;
        for (const Ciphertext &x : parts) p.push_back(&x);
        // checks and the allocation of the whole batch, copies of nothing yet
        const Ciphertext &p0 = *p.at(0);
        const Context &c = ev.context();
        size_t words = 0;
        uint32_t count = 0;
        for (const Ciphertext *q : p) {
            if (q->L != p0.L || q->size != p0.size || q->shared != p0.shared ||
                std::fabs(q->scale_ / p0.scale_ - 1.0) > 1e-12)
                throw Error("gather: parts differ in level, size or scale");
            words += q->polys() * q->L * c.n;
            count += q->count;
        }
        o.data = DeviceBuffer(c, words);
        o.count = count;
        o.size = p0.size;
        o.L = p0.L;
        o.scale_ = p0.scale_;
        o.shared = p0.shared;
    }
    const Context &c = ev.context();
    size_t off = 0;
    for (Ciphertext &x : parts) {
        const size_t w = x.polys() * x.L * c.n;
        c.check(shm_memcpy(c.handle(), o.data.data() + off, x.data.data(), w * 8, SHM_COPY_D2D, c.stream()));
        off += w;
        x = Ciphertext();
    }
    parts.clear();
    return o;
}

// LayerNorm over hidden columns packed one per ciphertext (layernorm, layernorm.cuh:899-):
// mean and variance are sums over the batch, the inverse square root is inv_sqrt_approx, and
// column i gets gamma_i (x_i - mean) / sqrt(var) + beta_i; 2 (d_newt + d_gold) + 8 levels
namespace {

// layernorm of x; with owned == &x's owner, x is released once the centred columns are formed
Ciphertext layernorm_impl(const Evaluator &ev, const Ciphertext &x, Ciphertext *owned, const std::vector<double> &gamma,
                          const std::vector<double> &beta, int d_newt, int d_gold, double var_scale) {
    need_ordinary(x, "layernorm");
    if (!(var_scale > 0)) throw Error("layernorm: var_scale must be positive");
    const uint32_t d = x.count;
    if (d == 0 || gamma.size() != d || beta.size() != d) throw Error("layernorm: gamma and beta need one value per column");
    const uint32_t need = 2 * (uint32_t)(d_newt + d_gold) + 9;
    if (x.L < need) throw Error("layernorm needs " + std::to_string(need) + " primes");
    const Context &c = ev.context();
    const double S = x.scale_;
    // columns are centred, squared and normalised in chunks, and the centred columns are kept as
    // chunks, so that at most a chunk's temporaries (and no broadcast of a whole batch) sit beside
    // them (at full width a whole-batch temporary is ~18 GB); the modular sums are the same
    const uint32_t chunk = std::min<uint32_t>(d, 128);
    const Ciphertext mean = ev.multiply_const(batch_sum(ev, x), 1.0 / d, S);
    std::vector<Ciphertext> xc;
    for (uint32_t lo = 0; lo < d; lo += chunk) {
        const uint32_t k = std::min(chunk, d - lo);
        xc.push_back(ev.sub(ev.mod_switch_to(ev.slice(x, lo, k), mean.L), batch_broadcast(ev, mean, k)));
    }
    if (owned) *owned = Ciphertext();
    Ciphertext sq_sum;
    for (const Ciphertext &part : xc) {
        Ciphertext s = batch_sum(ev, square(ev, part));
        sq_sum = sq_sum.count ? ev.add(sq_sum, s) : std::move(s);
    }
    const Ciphertext var = ev.multiply_const(sq_sum, var_scale / d, (double)c.primes[sq_sum.L - 2]);
    const Ciphertext inv = inv_sqrt_approx(ev, var, d_newt, d_gold);
    const double rs = std::sqrt(var_scale);
    std::vector<Ciphertext> cols;
    cols.reserve(d);
    uint32_t lo = 0;
    for (Ciphertext &part : xc) {
        const uint32_t k = part.count;
        const Ciphertext y = product(ev, part, batch_broadcast(ev, inv, k));
        part = Ciphertext();
        for (uint32_t i = 0; i < k; i++)
            cols.push_back(ev.add_const(ev.multiply_const(ev.slice(y, i, 1), gamma[lo + i] * rs, S), beta[lo + i]));
        lo += k;
    }
    return batch_gather(ev, std::move(cols));
}

}  // namespace

Ciphertext layernorm(const Evaluator &ev, const Ciphertext &x, const std::vector<double> &gamma,
                     const std::vector<double> &beta, int d_newt, int d_gold, double var_scale) {
    return layernorm_impl(ev, x, nullptr, gamma, beta, d_newt, d_gold, var_scale);
}

Ciphertext layernorm(const Evaluator &ev, Ciphertext &&x, const std::vector<double> &gamma,
                     const std::vector<double> &beta, int d_newt, int d_gold, double var_scale) {
    return layernorm_impl(ev, x, &x, gamma, beta, d_newt, d_gold, var_scale);
}

// softmax over the members of a batch (softmax.cuh:119-, without the attention layout's
// masks): e_i = exp_approx(x_i - shift), s = sum_scale * sum_i e_i brought into (0, 2) by the
// caller's sum_scale, y_i = sum_scale * e_i * inverse_approx(s, iter) = e_i / sum_j e_j;
// iter + 12 levels
Ciphertext softmax_batch(const Evaluator &ev, const Ciphertext &x, double shift, double sum_scale, int iter) {
    need_ordinary(x, "softmax");
    if (!(sum_scale > 0)) throw Error("softmax: sum_scale must be positive");
    const uint32_t need = (uint32_t)iter + 13;
    if (x.L < need) throw Error("softmax needs " + std::to_string(need) + " primes");
    const Context &c = ev.context();
    const double S = x.scale_;
    const Ciphertext e = exp_approx(ev, ev.add_const(x, -shift));
    const Ciphertext s = ev.multiply_const(batch_sum(ev, e), sum_scale, (double)c.primes[e.L - 2]);
    const Ciphertext inv = inverse_approx(ev, s, iter);
    const Ciphertext y = product(ev, e, gather_ptrs(ev, std::vector<const Ciphertext *>(x.count, &inv)));
    return ev.multiply_const(y, sum_scale, S);
}

namespace {

// member i of the batch gets the slot vector v_i added (encoded at the batch's level and scale;
// an empty vector adds nothing): c0 += encode(v_i) on every limb
Ciphertext add_slot_vectors(const Evaluator &ev, const Ciphertext &a, const std::vector<std::vector<double>> &v) {
    const Context &c = ev.context();
    Ciphertext o = ev.slice(a, 0, a.count);
    const size_t per = (size_t)a.size * a.L * c.n;
    for (uint32_t i = 0; i < a.count; i++) {
        if (v[i].empty()) continue;
        std::vector<cplx> z(v[i].begin(), v[i].end());
        const Plaintext p = ev.encoder().encode(z, a.L, a.scale_);
        uint64_t *c0 = o.data.data() + i * per;
        c.check(shm_add(c.handle(), c0, p.data.data(), c0, 1, a.L, c.stream()));
    }
    return o;
}

}  // namespace

// softmax of the attention block (softmax, softmax.cuh:119-): member i of the batch is shifted
// by -8.1 on the bias slots its position selects (all of them for i = 0; slots below
// num_batch (input_num - i) for 1 <= i <= input_num; none in the middle; slots from
// num_batch (num - i) on for i > num - input_num), exponentiated, and has 1 taken off every
// slot except those same bias slots; the members' sum is inverted (inverse_approx, iter) and
// multiplies each member.  num_batch = slots / 128.  iter + 10 levels.
Ciphertext softmax_attention(const Evaluator &ev, const Ciphertext &x, const std::vector<int> &bias_vec,
                             int input_num, int iter) {
    need_ordinary(x, "softmax");
    const uint32_t need = (uint32_t)iter + 11;
    if (x.L < need) throw Error("softmax needs " + std::to_string(need) + " primes");
    const Ciphertext e = softmax_attention_numerators(ev, x, bias_vec, input_num);
    return softmax_attention_finish(ev, e, batch_sum(ev, e), iter);
}

// the members' sum inverted (inverse_approx, iter steps) and multiplied into every member
Ciphertext softmax_attention_finish(const Evaluator &ev, const Ciphertext &e, const Ciphertext &sum, int iter) {
    need_ordinary(e, "softmax");
    if (sum.count != 1) throw Error("softmax: one sum ciphertext");
    const Ciphertext inv = inverse_approx(ev, sum, iter);
    return product(ev, e, gather_ptrs(ev, std::vector<const Ciphertext *>(e.count, &inv)));
}

Ciphertext softmax_attention_numerators(const Evaluator &ev, const Ciphertext &x, const std::vector<int> &bias_vec,
                                        int input_num) {
    need_ordinary(x, "softmax");
    const Context &c = ev.context();
    const size_t slots = c.n / 2;
    if (bias_vec.size() != slots) throw Error("softmax: bias_vec needs one entry per slot");
    if (x.L < 9) throw Error("softmax's exp needs 8 levels and one prime for its output");
    const int num = (int)x.count, nb = (int)(slots / 128);
    // which bias slots member i treats as its own: all (i = 0), a prefix, none, or a suffix
    auto selected = [&](int i, size_t s) {
        if (bias_vec[s] != 1) return false;
        if (i == 0) return true;
        if (i > input_num && i <= num - input_num) return false;
        if (i <= input_num) return (long long)s < (long long)nb * (input_num - i);
        return (long long)s >= (long long)(num - i) * nb;
    };
    std::vector<std::vector<double>> shift(num), sub(num);
    for (int i = 0; i < num; i++) {
        std::vector<double> sh(slots, 0.0), sb(slots, -1.0);
        bool any = false;
        for (size_t s = 0; s < slots; s++)
            if (selected(i, s)) {
                sh[s] = -8.1;
                sb[s] = 0.0;
                any = true;
            }
        if (any) shift[i] = std::move(sh);
        sub[i] = std::move(sb);
    }
    return add_slot_vectors(ev, exp_approx(ev, add_slot_vectors(ev, x, shift)), sub);
}

}  // namespace shmoai
