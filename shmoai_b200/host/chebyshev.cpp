// Chebyshev-series evaluation on ciphertext batches: the bootstrapper's EvalMod and the
// polynomial operators of the BERT layer (the reference's non_linear_func/, e.g. gelu_cheb,
// src/include/source/non_linear_func/gelu_other.cuh:258-300).
#include <cmath>

#include "internal.hpp"

namespace shmoai {
namespace detail {

// p = q T_m + r for Chebyshev coefficients c (degree < 2m)
void cheb_divide(const std::vector<double> &c, int m, std::vector<double> &q, std::vector<double> &r) {
    const int d = (int)c.size() - 1;
    q.assign(1, c[m]);
    for (int j = 1; j <= d - m; j++) q.push_back(2.0 * c[m + j]);
    r.assign(c.begin(), c.begin() + m);
    for (int j = 1; j <= d - m; j++) r[m - j] -= c[m + j];
}

int bitlen(uint32_t d) { return d ? 32 - __builtin_clz(d) : 0; }

// T_1 .. T_8 and T_16, T_32, ... by products 2 T_a T_b - T_{a-b}; each product is
// relinearised and rescaled in one ModDown by q_{L-1} P
ChebBasis cheb_basis(const Evaluator &ev, const Ciphertext &x, int deg) {
    ChebBasis T;
    T.emplace(1, ev.adjust(x, x.L, x.scale_));
    auto prod = [&](int a, int b) {
        Ciphertext p = ev.multiply_int(ev.relinearize_rescale(ev.multiply_lazy(T.at(a), T.at(b))), 2);
        if (a == b) return ev.add_const(p, -1.0);
        return ev.sub(p, ev.adjust(T.at(a - b), p.L, p.scale_));
    };
    const int g = 8;
    for (int k = 2; k <= g && k <= deg; k++) {
        if (k % 2 == 0) {
            T.emplace(k, prod(k / 2, k / 2));
        } else {
            const int a = 1 << (bitlen((uint32_t)k) - 1);
            T.emplace(k, prod(a, k - a));
        }
    }
    for (int m = 2 * g; m <= deg; m *= 2) T.emplace(m, prod(m / 2, m / 2));
    return T;
}

bool cheb_feasible(const ChebBasis &T, int ncoef, uint32_t lvl) {
    const int d = ncoef - 1;
    if (d < 8) {
        for (int i = 1; i <= d; i++)
            if (T.at(i).L < lvl + 1) return false;
        return true;
    }
    const int m = 1 << (bitlen((uint32_t)d) - 1);
    return T.at(m).L >= lvl + 1 && cheb_feasible(T, d - m + 1, lvl + 1) && cheb_feasible(T, m, lvl);
}

// sum_i c_i T_i, output at exactly scale S and lvl primes (baby-step giant-step).  A
// giant-step product is only added to, so it stays unrelinearised (size 3) through its
// rescale and the sum; the sum is relinearised once, where it is needed as a multiplicand
// or at the top (lazy = false), instead of every product on its own: two relinearisations
// fewer at degree 47.  A constant quotient multiplies T_m as a scalar.
Ciphertext cheb_eval(const Evaluator &ev, const ChebBasis &T, const std::vector<double> &c, double S, uint32_t lvl,
                     bool lazy) {
    const Context &ctx = ev.context();
    const int d = (int)c.size() - 1;
    if (d < 1) throw Error("Chebyshev piece of degree 0");
    if (d < 8) {
        // c_0 + sum_i c_i T_i with each term at scale S q: weight round(c_i S q / scale(T_i)),
        // one linear-combination pass (T_i read at their first lvl + 1 limbs), then the rescale
        const double q = (double)ctx.primes[lvl];
        std::vector<const Ciphertext *> X;
        std::vector<double> w;
        for (int i = 1; i <= d; i++) {
            X.push_back(&T.at(i));
            w.push_back(std::nearbyint(c[i] * (S * q / T.at(i).scale_)));
        }
        Ciphertext acc = ev.linear_combination(X, w, std::nearbyint(c[0] * (S * q)), lvl + 1, S * q);
        Ciphertext out = ev.rescale_to_next(acc);
        out.scale_ = S;
        return out;
    }
    const int m = 1 << (bitlen((uint32_t)d) - 1);
    std::vector<double> qc, rc;
    cheb_divide(c, m, qc, rc);
    Ciphertext Tm = ev.mod_switch_to(T.at(m), lvl + 1);
    Ciphertext prod;
    if (qc.size() == 1) {
        prod = ev.multiply_const(Tm, qc[0], S);  // scalar times T_m, rescaled to lvl primes at S
    } else {
        const double Sq = S * (double)ctx.primes[lvl] / Tm.scale_;
        Ciphertext qct = cheb_eval(ev, T, qc, Sq, lvl + 1);  // a multiplicand: relinearised
        prod = ev.rescale_to_next(ev.multiply_lazy(qct, Tm));
        prod.scale_ = S;
    }
    Ciphertext sum = ev.add(prod, cheb_eval(ev, T, rc, S, lvl, true));
    return lazy || sum.size == 2 ? std::move(sum) : ev.relinearize(sum);
}

}  // namespace detail

std::vector<double> chebyshev_interpolant(const std::function<double(double)> &f, double lo, double hi, int deg) {
    if (deg < 1 || !(hi > lo)) throw Error("Chebyshev interpolant needs deg >= 1 and lo < hi");
    const int m = deg + 1;
    std::vector<double> fx(m), c(m, 0.0);
    for (int k = 0; k < m; k++) fx[k] = f(0.5 * (hi + lo) + 0.5 * (hi - lo) * std::cos(M_PI * (k + 0.5) / m));
    for (int j = 0; j < m; j++) {
        double s = 0;
        for (int k = 0; k < m; k++) s += fx[k] * std::cos(M_PI * j * (k + 0.5) / m);
        c[j] = (j ? 2.0 : 1.0) * s / m;
    }
    return c;
}

Ciphertext evaluate_chebyshev(const Evaluator &ev, const Ciphertext &x, const std::vector<double> &c, double lo,
                              double hi) {
    if (x.shared || x.size != 2) throw Error("Chebyshev evaluation takes ordinary size-2 ciphertexts");
    if (c.size() < 2) throw Error("Chebyshev series of degree 0");
    if (!(hi > lo)) throw Error("Chebyshev interval needs lo < hi");
    const int deg = (int)c.size() - 1;
    // u = a x + b maps [lo, hi] onto [-1, 1]; one level for the scalar product, whose output
    // scale is set to the prime the next product is rescaled by, so the basis products keep
    // their scales near the primes whatever the input's scale
    const double a = 2.0 / (hi - lo), b = -(hi + lo) / (hi - lo);
    if (x.L < 3) throw Error("no level left for a Chebyshev series");
    // the basis's depth: T_2 one level, T_3..T_4 two, T_5..T_8 three, T_16 four, ...; its
    // deepest member must keep two primes (one for the leaves' rescale, one for the output)
    const std::string short_msg = "not enough levels for a Chebyshev series of degree " + std::to_string(deg);
    int depth = detail::bitlen((uint32_t)((deg < 8 ? deg : 8) - 1));
    for (int m = 16; m <= deg; m *= 2) depth = detail::bitlen((uint32_t)(m - 1));
    if ((int)x.L - 1 - depth < 2) throw Error(short_msg);
    Ciphertext u = ev.add_const(ev.multiply_const(x, a, (double)ev.context().primes[x.L - 2]), b);
    detail::ChebBasis T = detail::cheb_basis(ev, u, deg);
    uint32_t lvl = u.L - 1;
    while (!detail::cheb_feasible(T, deg + 1, lvl)) {
        if (lvl <= 1) throw Error(short_msg);
        lvl--;
    }
    return detail::cheb_eval(ev, T, c, x.scale_, lvl);
}

double gelu_exact(double x) { return 0.5 * x * (1.0 + std::erf(x / std::sqrt(2.0))); }

// The degree-24 GELU series of gelu_cheb (src/include/source/non_linear_func/gelu_other.cuh:
// 284-296): near-minimax on [-19.5, 12.5] in the variable u = (x + 3.5) / 16, max error 0.037
// there.  The same table, so that the operator computes the reference's polynomial.
const std::vector<double> &gelu_series() {
    static const std::vector<double> d = {
        3.4550752799e+00,  5.7852067632e+00,  3.1727714170e+00,  7.0234932500e-01,  -4.6200569546e-01,
        -3.7817535966e-01, 8.4136420694e-02,  2.2427456987e-01,  2.9451916291e-02,  -1.2928072669e-01,
        -6.6659430283e-02, 6.4349502364e-02,  7.1733295078e-02,  -1.9882581810e-02, -6.1145844240e-02,
        -8.4827295421e-03, 4.3597254356e-02,  2.3373027950e-02,  -2.4790187963e-02, -2.7940100474e-02,
        8.8404026343e-03,  2.3776567058e-02,  8.8171887083e-03,  -4.6290425955e-02, -9.7997267900e-03};
    return d;
}

Ciphertext gelu(const Evaluator &ev, const Ciphertext &x) { return evaluate_chebyshev(ev, x, gelu_series(), -19.5, 12.5); }

}  // namespace shmoai

namespace shmoai {

std::unique_ptr<Graph> capture_chebyshev(const Evaluator &ev, const Ciphertext &in, const std::vector<double> &c,
                                         double lo, double hi, Ciphertext &out) {
    // the output's shape from one run on the base evaluator; the buffer belongs to the base context
    Ciphertext shape = evaluate_chebyshev(ev, in, c, lo, hi);
    const Context &ctx = ev.context();
    out.data = DeviceBuffer(ctx, shape.data.words());
    out.count = shape.count;
    out.size = shape.size;
    out.L = shape.L;
    out.scale_ = shape.scale_;
    out.shared = shape.shared;
    ctx.synchronize();
    uint64_t *dst = out.data.data();
    const size_t bytes = shape.data.words() * 8;
    return std::unique_ptr<Graph>(new Graph(ev, [&in, c, lo, hi, dst, bytes](const Evaluator &e) {
        Ciphertext r = evaluate_chebyshev(e, in, c, lo, hi);
        const Context &v = e.context();
        v.check(shm_memcpy(v.handle(), dst, r.data.data(), bytes, SHM_COPY_D2D, v.stream()));
    }));
}

}  // namespace shmoai
