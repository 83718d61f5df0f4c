// S2C-first CKKS bootstrapping over ciphertext batches, ordinary and shared-a
// (the reference's BatchBootstrapper::bootstrap_ordinary_s2c_first and
// bootstrap_shared_a_s2c_first, src/include/source/bootstrapping/BatchBootstrap.cuh:674-819).
//
// Pipeline (input at `input_level` primes):
//   [shared-a: FmtSwitch forward of groups of n]
//   SlotToCoeff: 3 BSGS layers (input_level -> input_level - 3 primes), factor F on the last
//   ModRaise: 1 -> nq primes, scale := q0
//   CoeffToSlot: 3 BSGS layers (nq -> nq - 2 primes, the last NOT rescaled), 1/(2K) folded
//     into the first
//   conjugation split re = w + conj w, im = -i (w - conj w), run before the last rescale
//     so the key switch's low-frequency noise is divided by that prime
//   [shared-a: FmtSwitch backward of re and im]
//   rescale, EvalMod on re and im as one batch: Chebyshev interpolant of
//     cos(2 pi (K x - 1/4) / 2^r), degree 47, K = 25, r = 3 double angles -> sin(2 pi t);
//     the constant c_fin = q0 / (2 pi Delta F) and the scale Delta are reached through
//     exact scale targets, not an extra level
//   recombination re + i im (i = the monomial X^(N/2), free).
//
// Slot transforms: the slot-to-coefficient map V (V_jk = omega_j^k, slot order 5^j)
// factors, after a bit reversal that both directions absorb, into log2(n) radix-2
// butterfly stages (the special FFT of thirdparty/phantom-fhe/src/fft.cu:358-439);
// stages are grouped 5/5/5 for n = 2^15 (the reference's logn/3 split,
// BatchBootstrap.cuh:84-88) into three sparse matrices of <= 63 diagonals, applied by
// baby-step giant-step with pre-rotated diagonals: one hoisted ModUp for all baby steps,
// one multiply-plain-accumulate launch per giant step, one rescale per layer.  The
// diagonal plaintexts are encoded once and stay resident on the device (the reference
// re-encodes them on every call, SharedACoeffToSlot.cu:50-57).
//
// EvalMod uses a Chebyshev interpolant (degree 47) with three double angles where the
// reference uses an NTL Remez fit of degree 59 with two (ModularReducer.cu:40-54); with
// two double angles the interpolant leaves ~2e-7 error, too much for the 2e-5 target
// after the x512 amplitude correction, with three ~1e-13.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <set>

#include "internal.hpp"

namespace shmoai {

namespace {

using Vec = std::vector<cplx>;
using Diags = std::map<uint32_t, Vec>;  // offset mod n -> diagonal: (D x)_a = sum_d D_d[a] x_{a+d}

void accumulate(Diags &D, uint32_t k, const Vec &v) {
    auto it = D.find(k);
    if (it == D.end()) {
        D.emplace(k, v);
        return;
    }
    for (size_t i = 0; i < v.size(); i++) it->second[i] += v[i];
}

// out[i] = v[(i - shift) mod n]
Vec roll(const Vec &v, int64_t shift) {
    const int64_t n = (int64_t)v.size();
    const int64_t s = ((shift % n) + n) % n;
    Vec out(v.size());
    for (int64_t i = 0; i < n; i++) out[(i + s) % n] = v[i];
    return out;
}

Vec apply_diags(const Diags &D, const Vec &x) {
    Vec out(x.size(), cplx(0, 0));
    const size_t n = x.size();
    for (auto &kv : D)
        for (size_t a = 0; a < n; a++) out[a] += kv.second[a] * x[(a + kv.first) % n];
    return out;
}

struct Twiddles {
    uint32_t n, M;
    std::vector<uint64_t> rot;  // 5^j mod 4n
    std::vector<cplx> ksi;      // exp(2 pi i k / 4n)
    explicit Twiddles(uint32_t n_) : n(n_), M(4 * n_), rot(n_), ksi(4 * n_) {
        uint64_t e = 1;
        for (uint32_t j = 0; j < n; j++) {
            rot[j] = e;
            e = (e * 5) % M;
        }
        for (uint32_t k = 0; k < M; k++) {
            const double ang = 2.0 * M_PI * (double)k / (double)M;
            ksi[k] = cplx(std::cos(ang), std::sin(ang));
        }
    }
    // twiddle of the butterfly with half-width h at position a (lower partner's value)
    cplx t(uint32_t h, uint32_t a) const {
        const uint32_t ln = 2 * h, j = a % ln, jj = j < h ? j : j - h;
        return ksi[(rot[jj] % (4 * (uint64_t)ln)) * (M / (4 * ln))];
    }
};

// butterfly stages S_1 .. S_log2(n) with V R^-1 = S_log2(n) ... S_1
std::vector<Diags> special_fft_stages(const Twiddles &tw) {
    const uint32_t n = tw.n;
    std::vector<Diags> stages;
    for (uint32_t ln = 2; ln <= n; ln *= 2) {
        const uint32_t h = ln / 2;
        Vec d0(n), dp(n), dm(n);
        for (uint32_t a = 0; a < n; a++) {
            const bool lower = (a % ln) < h;
            const cplx t = tw.t(h, a);
            d0[a] = lower ? cplx(1, 0) : -t;
            dp[a] = lower ? t : cplx(0, 0);
            dm[a] = lower ? cplx(0, 0) : cplx(1, 0);
        }
        Diags D;
        accumulate(D, 0, d0);
        accumulate(D, h % n, dp);
        accumulate(D, (n - h) % n, dm);
        stages.push_back(std::move(D));
    }
    return stages;
}

// inverse of the stage with half-width h: x_a = (y_a + y_{a+h}) / 2, x_{a+h} = (y_a - y_{a+h}) / (2 t_a)
Diags inverse_stage(const Twiddles &tw, uint32_t h) {
    const uint32_t n = tw.n;
    Vec d0(n), dp(n), dm(n);
    for (uint32_t a = 0; a < n; a++) {
        const bool lower = (a % (2 * h)) < h;
        const cplx inv2t = 1.0 / (2.0 * tw.t(h, a));
        d0[a] = lower ? cplx(0.5, 0) : -inv2t;
        dp[a] = lower ? cplx(0.5, 0) : cplx(0, 0);
        dm[a] = lower ? cplx(0, 0) : inv2t;
    }
    Diags D;
    accumulate(D, 0, d0);
    accumulate(D, h % n, dp);
    accumulate(D, (n - h) % n, dm);
    return D;
}

// diagonals of P Q (Q applied first): (PQ)_{d+e} += P_d * Rot_d(Q_e)
Diags compose(const Diags &P, const Diags &Q, uint32_t n) {
    Diags out;
    for (auto &pd : P)
        for (auto &qe : Q) {
            const uint32_t k = (pd.first + qe.first) % n;
            Vec v(n);
            for (uint32_t a = 0; a < n; a++) v[a] = pd.second[a] * qe.second[(a + pd.first) % n];
            accumulate(out, k, v);
        }
    for (auto it = out.begin(); it != out.end();) {
        double mx = 0;
        for (auto &z : it->second) mx = std::max(mx, std::abs(z));
        it = mx > 0 ? std::next(it) : out.erase(it);
    }
    return out;
}

std::vector<uint32_t> layer_split(uint32_t logn) {
    const uint32_t d1 = logn / 3, d2 = (logn - d1) / 2;
    return {d1, d2, logn - d1 - d2};
}

// three grouped layers A, B, C with V R^-1 = C B A (A applied first)
std::vector<Diags> s2c_layers(const Twiddles &tw) {
    std::vector<Diags> st = special_fft_stages(tw);
    const uint32_t logn = (uint32_t)st.size();
    std::vector<Diags> out;
    uint32_t i = 0;
    for (uint32_t size : layer_split(logn)) {
        Diags M = st[i];
        for (uint32_t k = i + 1; k < i + size; k++) M = compose(st[k], M, tw.n);
        out.push_back(std::move(M));
        i += size;
    }
    return out;
}

// three grouped layers with (V R^-1)^-1 = A^-1 B^-1 C^-1 (C^-1 applied first)
std::vector<Diags> c2s_layers(const Twiddles &tw) {
    const uint32_t logn = (uint32_t)std::lround(std::log2((double)tw.n));
    std::vector<Diags> inv;
    for (uint32_t k = 0; k < logn; k++) inv.push_back(inverse_stage(tw, 1u << k));
    std::vector<std::vector<uint32_t>> groups;
    uint32_t i = 0;
    for (uint32_t size : layer_split(logn)) {
        std::vector<uint32_t> g;
        for (uint32_t k = i; k < i + size; k++) g.push_back(k);
        groups.push_back(g);
        i += size;
    }
    std::vector<Diags> out;
    for (auto g = groups.rbegin(); g != groups.rend(); ++g) {
        Diags M = inv[g->back()];
        for (auto k = g->rbegin() + 1; k != g->rend(); ++k) M = compose(inv[*k], M, tw.n);
        out.push_back(std::move(M));
    }
    return out;
}

// Chebyshev interpolant of f(K x) on [-1, 1] at the deg + 1 Chebyshev nodes
std::vector<double> cheb_interp(double (*f)(double, int), int r, double K, int deg) {
    const int m = deg + 1;
    std::vector<double> fx(m), c(m, 0.0);
    for (int k = 0; k < m; k++) fx[k] = f(K * std::cos(M_PI * (k + 0.5) / m), r);
    for (int j = 0; j < m; j++) {
        double s = 0;
        for (int k = 0; k < m; k++) s += fx[k] * std::cos(M_PI * j * (k + 0.5) / m);
        c[j] = (j ? 2.0 : 1.0) * s / m;
    }
    return c;
}

double evalmod_target(double t, int r) { return std::cos(2.0 * M_PI * (t - 0.25) / std::ldexp(1.0, r)); }


int64_t floordiv(int64_t a, int64_t b) {
    int64_t q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) q--;
    return q;
}

// the diagonal offsets of a layer in units of their gcd b, centred to (-span/2, span/2]
std::map<int64_t, const Vec *> centred_offsets(const Diags &diags, int64_t slots, int64_t &b) {
    b = 0;
    for (auto &kv : diags) b = std::gcd(b, (int64_t)kv.first);
    if (!b) b = 1;
    const int64_t span = slots / b;
    std::map<int64_t, const Vec *> ts;
    for (auto &kv : diags) {
        int64_t t = (int64_t)kv.first / b;
        if (t > span / 2) t -= span;
        ts[t] = &kv.second;
    }
    return ts;
}

int64_t default_g1(size_t diagonals) {
    return (int64_t)1 << (int)std::ceil(std::log2(std::sqrt((double)diagonals)));
}

// nonzero baby steps v and giant steps u of the split t = g1 u + v
void split_counts(const std::map<int64_t, const Vec *> &ts, int64_t g1, size_t &baby, size_t &giant) {
    std::set<int64_t> us, vs;
    for (auto &kv : ts) {
        const int64_t u = floordiv(kv.first, g1);
        us.insert(u);
        vs.insert(kv.first - u * g1);
    }
    baby = vs.size() - vs.count(0);
    giant = us.size() - us.count(0);
}

}  // namespace

// ------------------------------------------------------------------ LinearTransform

// sum_d D_d * Rot_d(x) at one level by baby-step giant-step: offsets t (in units of
// the gcd b) split as t = g1 u + v; baby steps Rot_{v b}(x) share one hoisted ModUp,
// diagonals are pre-rotated by -g1 u b, so each giant step is one rotation of
// sum_v Rot_{-g1 u b}(D_t) * Rot_{v b}(x).
class LinearTransform {
   public:
    // g1 = baby-step count (0: default_g1)
    LinearTransform(const Evaluator &ev, const Diags &diags, uint32_t level, int64_t g1 = 0) : level_(level) {
        const Context &c = ev.context();
        const std::map<int64_t, const Vec *> ts = centred_offsets(diags, c.n / 2, b_);
        g1_ = g1 > 0 ? g1 : default_g1(ts.size());
        pt_scale_ = (double)c.primes[level - 1];
        for (auto &kv : ts) {
            const int64_t u = floordiv(kv.first, g1_), v = kv.first - u * g1_;
            Vec P = roll(*kv.second, g1_ * u * b_);
            // over QlP when the context has special primes: the first `level` limbs serve ordinary
            // batches, all of them the double-hoisted shared-a path (apply_ext)
            groups_[u].emplace_back(v, c.np ? ev.encoder().encode_ext(P, level, pt_scale_)
                                            : ev.encoder().encode(P, level, pt_scale_));
        }
        std::set<int64_t> bs;
        for (auto &g : groups_)
            for (auto &vp : g.second) bs.insert(vp.first);
        baby_.assign(bs.begin(), bs.end());
    }

    std::set<int> steps() const {
        std::set<int> s;
        for (int64_t v : baby_)
            if (v) s.insert((int)(v * b_));
        for (auto &g : groups_)
            if (g.first) s.insert((int)(g1_ * g.first * b_));
        return s;
    }

    Ciphertext apply(const Evaluator &ev, const Ciphertext &x, bool rescale = true) const {
        const Ciphertext *xp = &x;
        Ciphertext dropped;
        if (x.L != level_) {
            dropped = ev.mod_switch_to(x, level_);
            xp = &dropped;
        }
        if (ev.context().np && (xp->shared || xp->size == 2)) return apply_ext(ev, *xp, rescale);
        std::vector<int> bsteps;
        for (int64_t v : baby_)
            if (v) bsteps.push_back((int)(v * b_));
        std::map<int, Ciphertext> rot = ev.rotate_many(*xp, bsteps);
        Ciphertext acc;
        bool have = false;
        for (auto &g : groups_) {
            std::vector<const Ciphertext *> X;
            std::vector<const Plaintext *> P;
            for (auto &vp : g.second) {
                X.push_back(vp.first ? &rot.at((int)(vp.first * b_)) : xp);
                P.push_back(&vp.second);
            }
            Ciphertext inner = ev.multiply_plain_accumulate(X, P);
            inner.scale_ = xp->scale_ * pt_scale_;
            if (g.first) inner = ev.rotate_vector(inner, (int)(g1_ * g.first * b_));
            if (!have) {
                acc = std::move(inner);
                have = true;
            } else {
                acc = ev.add(acc, inner);
            }
        }
        return rescale ? ev.rescale_to_next(acc) : std::move(acc);
    }

   private:
    // Double hoisting (Bossuat et al.): the baby-step rotations stay in the extended basis QlP
    // (no ModDown), the inner sums multiply QlP plaintexts, each giant step brings only its a
    // row down before rotating, the giant-step results add up in QlP and one ModDown of every
    // row ends the layer.  Every extended batch stands for its ModDown, so the result is the
    // layer's product up to ModDown rounding (a few units).  Shared-a groups of n use their
    // Sh-Galois keys; an ordinary batch is the case n = 1 (an ordinary Galois key has the
    // one-member Sh-Galois layout [dnum][2][QP][N]).
    Ciphertext apply_ext(const Evaluator &ev, const Ciphertext &x, bool rescale) const {
        const Context &c = ev.context();
        shm_context *h = c.handle();
        const std::map<uint32_t, DeviceBuffer> *table = nullptr;
        if (x.shared) {
            if (!ev.shared_keys || ev.shared_keys->members != x.members())
                throw Error("no shared-a keys for this group size");
            table = &ev.shared_keys->galois;
        } else {
            if (!ev.galois_keys) throw Error("no Galois keys");
            table = ev.galois_keys;
        }
        const uint32_t G = x.count, n = x.shared ? x.members() : 1, H = n + 1, L = level_;
        const size_t E = (size_t)G * H * (L + c.np) * c.n;  // words of one extended batch
        auto key_of = [&](int64_t step) {
            const uint32_t elt = ev.galois_elt((int)step);
            auto it = table->find(elt);
            if (it == table->end()) throw Error("missing Galois key for element " + std::to_string(elt));
            return std::make_pair(elt, (const uint64_t *)it->second.data());
        };
        const size_t wsb = std::max(shm_shared_rotate_ext_workspace_bytes(h, G, n, L),
                                    shm_moddown_ext_workspace_bytes(h, G * H, L));
        DeviceBuffer ws(c, wsb / 8 + 1);
        // baby steps, one ModUp for all of them
        std::vector<int64_t> babies;
        for (int64_t v : baby_)
            if (v) babies.push_back(v);
        DeviceBuffer rots(c, E * babies.size());
        std::map<int64_t, const uint64_t *> ext_of;
        {
            std::vector<uint32_t> elts;
            std::vector<const uint64_t *> keys;
            std::vector<uint64_t *> outs;
            for (size_t i = 0; i < babies.size(); i++) {
                auto k = key_of(babies[i] * b_);
                elts.push_back(k.first);
                keys.push_back(k.second);
                outs.push_back(rots.data() + i * E);
                ext_of[babies[i]] = outs.back();
            }
            if (!babies.empty())
                c.check(shm_shared_rotate_ext(h, x.data.data(), 0, G, n, (uint32_t)babies.size(), elts.data(),
                                              keys.data(), outs.data(), L, ws.data(), ws.words() * 8, c.stream()));
        }
        DeviceBuffer xext(c, E);
        c.check(shm_extend(h, x.data.data(), xext.data(), G * H, L, c.stream()));
        ext_of[0] = xext.data();
        DeviceBuffer total, inner(c, E), rot(c, E);
        for (auto &g : groups_) {
            std::vector<const uint64_t *> X, P;
            for (auto &vp : g.second) {
                X.push_back(ext_of.at(vp.first));
                P.push_back(vp.second.data.data());
            }
            c.check(shm_multiply_plain_accumulate_ext(h, X.data(), P.data(), (uint32_t)X.size(), inner.data(), G * H,
                                                      L, 0, c.stream()));
            DeviceBuffer *term = &inner;
            if (g.first) {
                auto k = key_of(g1_ * g.first * b_);
                uint64_t *o = rot.data();
                c.check(shm_shared_rotate_ext(h, inner.data(), 1, G, n, 1, &k.first, &k.second, &o, L, ws.data(),
                                              ws.words() * 8, c.stream()));
                term = &rot;
            }
            if (!total.data()) {
                std::swap(total, *term);
                if (!inner.data()) inner = DeviceBuffer(c, E);
                if (!rot.data()) rot = DeviceBuffer(c, E);
            } else {
                c.check(shm_add_ext(h, total.data(), term->data(), total.data(), G * H, L, c.stream()));
            }
        }
        Ciphertext out;
        out.data = DeviceBuffer(c, (size_t)G * H * L * c.n);
        out.count = G;
        out.size = H;
        out.L = L;
        out.scale_ = x.scale_ * pt_scale_;
        out.shared = x.shared;
        c.check(shm_moddown_ext(h, total.data(), out.data.data(), G * H, L, ws.data(), ws.words() * 8, c.stream()));
        return rescale ? ev.rescale_to_next(out) : std::move(out);
    }

    uint32_t level_;
    int64_t b_ = 1, g1_ = 1;
    double pt_scale_ = 1;
    std::map<int64_t, std::vector<std::pair<int64_t, Plaintext>>> groups_;  // u -> (v, pre-rotated diagonal)
    std::vector<int64_t> baby_;
};

// ------------------------------------------------------------------ BatchBootstrapper

BatchBootstrapper::BatchBootstrapper(Evaluator &ev, BootstrapParams p) : ev_(ev), p_(p) {}

BatchBootstrapper::~BatchBootstrapper() {
    for (auto *lt : s2c_) delete lt;
    for (auto *lt : c2s_) delete lt;
    for (auto *lt : s2c_late_) delete lt;
}

void BatchBootstrapper::prepare() {
    const Context &c = ev_.context();
    if (p_.input_level < 4 || p_.input_level > c.nq) throw Error("input level must be in [4, nq]");
    for (auto *lt : s2c_) delete lt;
    for (auto *lt : c2s_) delete lt;
    {
        std::lock_guard<std::mutex> g(late_mu_);
        for (auto *lt : s2c_late_) delete lt;
        s2c_late_.clear();
    }
    s2c_.clear();
    c2s_.clear();
    const Twiddles tw(c.n / 2);
    std::vector<Diags> s = s2c_layers(tw);
    for (auto &kv : s[2])
        for (auto &z : kv.second) z *= p_.F;
    for (uint32_t i = 0; i < 3; i++) s2c_.push_back(new LinearTransform(ev_, s[i], p_.input_level - i, p_.bsgs_g1[i]));
    std::vector<Diags> ci = c2s_layers(tw);
    for (auto &kv : ci[0])
        for (auto &z : kv.second) z /= 2.0 * p_.K;
    for (uint32_t i = 0; i < 3; i++) c2s_.push_back(new LinearTransform(ev_, ci[i], c.nq - i, p_.bsgs_g1[3 + i]));
    top_ = c.nq;
    q0_ = (double)c.primes[0];
    cheb_ = cheb_interp(evalmod_target, p_.double_angles, p_.K, p_.degree);
    c_fin_ = q0_ / (2.0 * M_PI * p_.scale * p_.F);
    c.synchronize();  // the diagonals are read from other streams later
}

std::vector<int> BatchBootstrapper::rotation_steps() const {
    std::set<int> s;
    for (auto *lt : s2c_) {
        std::set<int> t = lt->steps();
        s.insert(t.begin(), t.end());
    }
    for (auto *lt : c2s_) {
        std::set<int> t = lt->steps();
        s.insert(t.begin(), t.end());
    }
    return std::vector<int>(s.begin(), s.end());
}

std::vector<uint32_t> BatchBootstrapper::galois_elts() const {
    std::set<uint32_t> e;
    for (int st : rotation_steps()) e.insert(ev_.galois_elt(st));
    e.insert(2 * ev_.context().n - 1);
    return std::vector<uint32_t>(e.begin(), e.end());
}

SharedAKeys BatchBootstrapper::prepare_shared_keys(KeyGenerator &kg, uint32_t members, uint32_t hw) const {
    return kg.shared_keys(members, galois_elts(), hw);
}


// x holds t / K; returns c_fin * sin(2 pi t) read at scale Delta.  Backward scale
// targets: the i-th double angle squares at level lvl - i and drops prime lvl - 1 - i,
// so s_in = sqrt(s_out * q); the last output scale is Delta * c_fin, which reads as the
// value c_fin * y at scale Delta.
Ciphertext BatchBootstrapper::evalmod(const Ciphertext &x, const Evaluator *evp) const {
    const Evaluator &ev = evp ? *evp : ev_;
    const Context &c = ev.context();
    const int deg = (int)cheb_.size() - 1;
    detail::ChebBasis T = detail::cheb_basis(ev, x, deg);
    uint32_t lvl = x.L - 1;
    while (!detail::cheb_feasible(T, deg + 1, lvl)) {
        if (lvl == 0) throw Error("not enough levels for EvalMod");
        lvl--;
    }
    double s = p_.scale * c_fin_;
    for (int i = p_.double_angles - 1; i >= 0; i--) s = std::sqrt(s * (double)c.primes[lvl - 1 - i]);
    Ciphertext y = detail::cheb_eval(ev, T, cheb_, s, lvl);
    for (int i = 0; i < p_.double_angles; i++) {  // y = 2 y^2 - 1, the affine part in one pass
        const Ciphertext sq = ev.relinearize_rescale(ev.multiply_lazy(y, y));
        y = ev.linear_combination({&sq}, {2.0}, std::nearbyint(-1.0 * sq.scale_), sq.L, sq.scale_);
    }
    y.scale_ /= c_fin_;
    return y;
}

void BatchBootstrapper::slots_to_re_im(const Evaluator &ev, Ciphertext x, Ciphertext &re, Ciphertext &im) const {
    if (s2c_.empty()) throw Error("call prepare() first");
    if (x.L != p_.input_level) throw Error("bootstrap input must have input_level primes");
    for (auto *lt : s2c_) x = lt->apply(ev, x);
    Ciphertext w = ev.mod_raise(x, top_);
    w.scale_ = q0_;
    w = c2s_[0]->apply(ev, w);
    w = c2s_[1]->apply(ev, w);
    w = c2s_[2]->apply(ev, w, false);
    Ciphertext wc = ev.complex_conjugate(w);
    re = ev.add(w, wc);
    im = ev.multiply_i(ev.sub(w, wc), -1);
}

Ciphertext BatchBootstrapper::finish(const Evaluator &ev, const Ciphertext &re, const Ciphertext &im) const {
    Ciphertext y = evalmod(ev.rescale_to_next(ev.concat(re, im)), &ev);
    const uint32_t nb = re.count;
    return ev.add(ev.slice(y, 0, nb), ev.multiply_i(ev.slice(y, nb, nb)));
}

Ciphertext BatchBootstrapper::bootstrap_ordinary_s2c_first(const Ciphertext &ct, const Evaluator *evp) const {
    const Evaluator &ev = evp ? *evp : ev_;
    if (ct.shared || ct.size != 2) throw Error("bootstrap takes ordinary size-2 ciphertexts");
    Ciphertext re, im;
    slots_to_re_im(ev, ev.adjust(ct, ct.L, ct.scale_), re, im);
    return finish(ev, re, im);
}

// C2S-first: the input's coefficients t = Delta c / q0 (c = the encoding of its slots) after ModRaise;
// CoeffToSlot and EvalMod leave c / F in the slots (EvalMod's c_fin assumes SlotToCoeff's factor F),
// and SlotToCoeff with F on its last layer puts Delta c back into the coefficients
Ciphertext BatchBootstrapper::bootstrap_c2s_first(const Ciphertext &ct, const Evaluator *evp) const {
    const Evaluator &ev = evp ? *evp : ev_;
    if (c2s_.empty()) throw Error("call prepare() first");
    if (ct.shared || ct.size != 2) throw Error("bootstrap takes ordinary size-2 ciphertexts");
    const Ciphertext x1 = ev.adjust(ct, 1, p_.scale);
    Ciphertext w = ev.mod_raise(x1, top_);
    w.scale_ = q0_;
    w = c2s_[0]->apply(ev, w);
    w = c2s_[1]->apply(ev, w);
    w = c2s_[2]->apply(ev, w, false);
    const Ciphertext wc = ev.complex_conjugate(w);
    Ciphertext y = finish(ev, ev.add(w, wc), ev.multiply_i(ev.sub(w, wc), -1));
    {
        std::lock_guard<std::mutex> g(late_mu_);
        if (s2c_late_.empty() || y.L != late_level_) {
            if (y.L < 4) throw Error("not enough levels left for SlotToCoeff after EvalMod");
            for (auto *lt : s2c_late_) delete lt;
            s2c_late_.clear();
            const Twiddles tw(ev.context().n / 2);
            std::vector<Diags> s = s2c_layers(tw);
            for (auto &kv : s[2])
                for (auto &z : kv.second) z *= p_.F;
            for (uint32_t i = 0; i < 3; i++)
                s2c_late_.push_back(new LinearTransform(ev_, s[i], y.L - i, p_.bsgs_g1[i]));
            late_level_ = y.L;
            ev_.context().synchronize();
        }
    }
    for (auto *lt : s2c_late_) y = lt->apply(ev, y);
    return y;
}

Ciphertext BatchBootstrapper::bootstrap_shared_a_s2c_first(const Ciphertext &ct, uint32_t members,
                                                           const Evaluator *evp) const {
    const Evaluator &ev = evp ? *evp : ev_;
    Ciphertext re, im;
    slots_to_re_im(ev, ev.to_shared(ct, members), re, im);
    return finish(ev, ev.from_shared(re), ev.from_shared(im));
}

// ------------------------------------------------------------------ autotuning

namespace {

// milliseconds of one hoisted rotation batch with k targets of `count` ciphertexts at L primes:
// one ModUp and k inner products with extended outputs, the rotation of the double-hoisted
// layers; an ordinary batch is groups of one member.  Uniform scratch residues and a scratch
// key (timing only)
double time_rotations(const Evaluator &ev, uint32_t count, uint32_t members, uint32_t L, uint32_t k) {
    const Context &c = ev.context();
    shm_context *h = c.handle();
    const uint32_t nm = members ? members : 1, H = nm + 1, units = count / nm, QP = c.nq + c.np;
    const size_t ln = (size_t)L * c.n;
    DeviceBuffer x(c, units * H * ln), key(c, (size_t)c.dnum * H * QP * c.n);
    c.check(shm_sample_uniform(h, x.data(), units * H, L, 0x7E5A, c.stream()));
    c.check(shm_sample_uniform(h, key.data(), c.dnum * H, QP, 0x7E5B, c.stream()));
    std::vector<DeviceBuffer> outs;
    std::vector<uint64_t *> optr;
    std::vector<const uint64_t *> keys(k, key.data());
    std::vector<uint32_t> elts;
    for (uint32_t i = 0; i < k; i++) {
        outs.emplace_back(c, (size_t)units * H * (L + c.np) * c.n);
        optr.push_back(outs.back().data());
        elts.push_back(ev.galois_elt((int)i + 1));
    }
    DeviceBuffer ws(c, shm_shared_rotate_ext_workspace_bytes(h, units, nm, L) / 8 + 1);
    auto run = [&] {
        c.check(shm_shared_rotate_ext(h, x.data(), 0, units, nm, k, elts.data(), keys.data(), optr.data(), L,
                                      ws.data(), ws.words() * 8, c.stream()));
    };
    run();
    c.synchronize();
    const int reps = 3;
    const auto t0 = std::chrono::steady_clock::now();
    for (int r = 0; r < reps; r++) run();
    c.synchronize();
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / reps;
}

}  // namespace

void BatchBootstrapper::set_split(const int g1[6]) {
    for (int i = 0; i < 6; i++) {
        if (g1[i] < 0) throw Error("BSGS split: baby-step counts must be >= 0");
        p_.bsgs_g1[i] = g1[i];
    }
    prepare();
}

std::vector<TuneRecord> BatchBootstrapper::tune(uint32_t count, uint32_t members) {
    const Context &c = ev_.context();
    shm_context *h = c.handle();
    if (!count || (members && count % members)) throw Error("tune: count must be a positive multiple of members");
    std::vector<TuneRecord> out;
    auto kernel_knob = [&](const char *name, int knob, uint32_t size, uint32_t level, uint32_t mem,
                           std::vector<std::string> names) {
        float t[8] = {0};
        uint32_t best = 0;
        c.check(shm_autotune(h, knob, size, level, mem, t, 8, &best));
        TuneRecord r{name, names, {}, best};
        for (size_t i = 0; i < names.size(); i++) r.ms.push_back(t[i]);
        out.push_back(r);
    };
    // EvalMod's key switches dominate: ~4096 limbs is one relinearisation's ModUp batch scale
    kernel_knob("ntt_tile", SHM_TUNE_NTT_TILE, std::min<uint32_t>(4096, 2 * count * c.nq), 0, 0,
                {"16 cols, 4 CTAs/SM", "16 cols, 3 CTAs/SM", "8 cols, 8 CTAs/SM", "8 cols, 6 CTAs/SM"});
    if (members)
        kernel_knob("ip_chunk", SHM_TUNE_IP_CHUNK, count / members, c.nq, members, {"16 KB", "32 KB", "64 KB", "96 KB"});
    // The plain transforms of the first knob hardly separate the tiles (within 0.5 % of each other), while the
    // bootstrap step ran 9 % faster with 8 CTAs/SM than with 6: its transforms are mostly the
    // ModUp- and ModDown-fused ones of key switches.  So the tile is chosen again by timing one
    // hoisted rotation of the batch at the top level, which runs those fused launches (where the
    // knob times real kernels: the host-only build reports zero for every candidate).
    if (*std::max_element(out.front().ms.begin(), out.front().ms.end()) > 0) {
        TuneRecord r{"ntt_tile (hoisted rotation, top level)", out.front().candidates, {}, 0};
        double best = 1e300;
        for (uint32_t v = 0; v < r.candidates.size(); v++) {
            c.check(shm_tune_set(h, SHM_TUNE_NTT_TILE, v));
            const double t = time_rotations(ev_, count, members, c.nq, 1);
            r.ms.push_back(t);
            if (t < best) {
                best = t;
                r.chosen = v;
            }
        }
        c.check(shm_tune_set(h, SHM_TUNE_NTT_TILE, (uint32_t)r.chosen));
        out.push_back(r);
    }

    // BSGS split per layer: cost(g1) = (1 + giant) ModUps + (baby + giant) per-step switches,
    // both timed at the layer's level (one and three targets of a hoisted batch)
    const Twiddles tw(c.n / 2);
    const std::vector<Diags> layers[2] = {s2c_layers(tw), c2s_layers(tw)};
    for (int layer = 0; layer < 6; layer++) {
        const uint32_t L = layer < 3 ? p_.input_level - layer : c.nq - (layer - 3);
        const double t1 = time_rotations(ev_, count, members, L, 1), t3 = time_rotations(ev_, count, members, L, 3);
        const double step = std::max(0.0, (t3 - t1) / 2), modup = std::max(0.0, t1 - step);
        int64_t b = 1;
        const auto ts = centred_offsets(layers[layer / 3][layer % 3], c.n / 2, b);
        TuneRecord r{"bsgs_g1[" + std::string(layer < 3 ? "S2C " : "C2S ") + std::to_string(layer % 3) + "] at " +
                         std::to_string(L) + " primes",
                     {}, {}, 0};
        double best = 1e300;
        for (int64_t g1 = 1; g1 <= (int64_t)ts.size() * 2; g1 *= 2) {
            size_t baby = 0, giant = 0;
            split_counts(ts, g1, baby, giant);
            const double cost = (1 + giant) * modup + (baby + giant) * step;
            r.candidates.push_back(std::to_string(g1));
            r.ms.push_back(cost);
            if (cost < best) {
                best = cost;
                r.chosen = r.candidates.size() - 1;
                p_.bsgs_g1[layer] = (int)g1;
            }
        }
        out.push_back(r);
    }
    prepare();
    return out;
}

double slot_transform_selfcheck(uint32_t log_slots) {
    const uint32_t n = 1u << log_slots, N = 2 * n, M = 2 * N;
    const Twiddles tw(n);
    Vec w(n);
    for (uint32_t i = 0; i < n; i++) {
        const double a = (double)(detail::mix64(7, 2 * i) >> 11) * 0x1.0p-53 - 0.5;
        const double b = (double)(detail::mix64(7, 2 * i + 1) >> 11) * 0x1.0p-53 - 0.5;
        w[i] = cplx(a, b);
    }
    std::vector<uint64_t> ex(n);
    uint64_t e = 1;
    for (uint32_t j = 0; j < n; j++) {
        ex[j] = e;
        e = (e * 5) % M;
    }
    Vec Vw(n, cplx(0, 0));
    double vmax = 0;
    for (uint32_t j = 0; j < n; j++) {
        for (uint32_t k = 0; k < n; k++) {
            const double ang = 2.0 * M_PI * (double)((ex[j] * k) % M) / (double)M;
            Vw[j] += w[k] * cplx(std::cos(ang), std::sin(ang));
        }
        vmax = std::max(vmax, std::abs(Vw[j]));
    }
    Vec y(n);
    for (uint32_t i = 0; i < n; i++) {
        uint32_t r = 0;
        for (uint32_t b = 0; b < log_slots; b++) r |= ((i >> b) & 1u) << (log_slots - 1 - b);
        y[i] = w[r];
    }
    const Vec wr = y;
    for (auto &L : s2c_layers(tw)) y = apply_diags(L, y);
    double err = 0;
    for (uint32_t j = 0; j < n; j++) err = std::max(err, std::abs(y[j] - Vw[j]) / vmax);
    Vec z = Vw;
    for (auto &L : c2s_layers(tw)) z = apply_diags(L, z);
    for (uint32_t j = 0; j < n; j++) err = std::max(err, std::abs(z[j] - wr[j]));
    return err;
}

}  // namespace shmoai
