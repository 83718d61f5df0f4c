// One BERT encoder layer under the MOAI column packing (src/include/test/test_single_layer.cuh:
// 422-2062 and src/include/source/att_block/single_att_block.cuh:21-315): the attention heads
// (QKV projections, QK^T in the column packing, the masked softmax with a bootstrap of its sum,
// softmax * V in the diagonal packing), SelfOutput, four bootstrap segments, two LayerNorms with
// their residual inputs, the Intermediate projection, GELU and the masked Final projection, with
// the reference's stage names and per-stage wall time.
//
// Level plan on the bootstrapping chain (35 ciphertext primes; bootstrap input at input_level = 4
// primes, output at `top` = 23 primes and scale Delta):
//   X (top) -> QKV (top - 1) -> QK^T (top - 2) -> exp (8 levels) ; sums -> bootstrap -> inverse
//   (iter + 1) -> times the numerators -> softmax * V (1) -> SelfOutput (1) -> Boot1 -> + X ->
//   LayerNorm1 (2 (newt + gold) + 8) -> Boot2 -> Intermediate at gelu_input + 1 -> GELU (6) ->
//   Final (masked, 2) -> Boot3 -> + H1 -> LayerNorm2 -> Boot4.
// Before a bootstrap a batch is brought to input_level primes at scale Delta (Evaluator::adjust:
// one level when its scale differs).  The B200 form batches where the reference loops: all
// projections are exact tensor-core contractions over the whole batch, the 12 heads' softmax sums
// are bootstrapped together, and each bootstrap segment runs the ciphertexts in batches (shared-a
// groups for the "sham" form); the "orig" form bootstraps one ciphertext per call.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <set>

#include "internal.hpp"

namespace shmoai {

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// weights [rows][cols] (row-major doubles) of columns [c0, c0 + n) -> integers at w_scale
std::vector<int64_t> int_weights(const std::vector<double> &W, uint32_t rows, uint32_t cols, uint32_t c0, uint32_t n,
                                 double w_scale, double factor = 1.0) {
    std::vector<int64_t> out((size_t)rows * n);
    for (uint32_t r = 0; r < rows; r++)
        for (uint32_t j = 0; j < n; j++)
            out[(size_t)r * n + j] = (int64_t)std::llround(W[(size_t)r * cols + c0 + j] * factor * w_scale);
    return out;
}

constexpr double kSoftmaxShift = -8.1;  // softmax.cuh's shift of the valid scores before exp

bool all_ones(const std::vector<int> &m) {
    return std::all_of(m.begin(), m.end(), [](int v) { return v == 1; });
}

}  // namespace

std::vector<int> bert_layer_rotation_steps(const BertLayerConfig &cfg, uint32_t slots) {
    const uint32_t nb = slots / cfg.tokens;
    std::vector<int> steps;
    for (uint32_t i = 1; i < cfg.tokens; i++) steps.push_back((int)(i * nb));
    return steps;
}

// column o of Y gets b[o] on the valid slots (the reference encodes the bias vector masked by
// bias_vec, single_att_block.cuh:54-70): a scalar add on every limb when every slot is valid,
// else one encoded slot vector per column (encoded in one batch on the device)
Ciphertext add_column_bias(const Evaluator &ev, const Ciphertext &Y, const std::vector<double> &b,
                           const std::vector<int> &mask) {
    if (b.size() != Y.count) throw Error("bias: one value per column");
    const Context &c = ev.context();
    if (mask.empty() || all_ones(mask)) {
        std::vector<Ciphertext> cols;
        cols.reserve(Y.count);
        for (uint32_t o = 0; o < Y.count; o++) cols.push_back(ev.add_const(ev.slice(Y, o, 1), b[o]));
        return batch_gather(ev, cols);
    }
    if (mask.size() != c.n / 2) throw Error("bias: the mask needs one entry per slot");
    std::vector<std::vector<cplx>> z(Y.count, std::vector<cplx>(c.n / 2));
    for (uint32_t o = 0; o < Y.count; o++)
        for (size_t s = 0; s < mask.size(); s++) z[o][s] = mask[s] ? cplx(b[o], 0) : cplx(0, 0);
    const size_t ln = (size_t)Y.L * c.n;
    DeviceBuffer coeffs(c, (size_t)Y.count * c.n), pt(c, Y.count * ln);
    ev.encoder().encode_rows(z, Y.scale_, coeffs.data());
    ev.encoder().lift(coeffs.data(), Y.count, Y.L, pt.data());
    Ciphertext o = ev.slice(Y, 0, Y.count);
    for (uint32_t i = 0; i < Y.count; i++) {
        uint64_t *c0 = o.data.data() + 2 * i * ln;
        c.check(shm_add(c.handle(), c0, pt.data() + i * ln, c0, 1, Y.L, c.stream()));
    }
    return o;
}

namespace {

Ciphertext bootstrap_segment_impl(const Evaluator &ev, const BatchBootstrapper &boot, const Ciphertext &x,
                                  Ciphertext *owned, uint32_t members, uint32_t batch) {
    const BootstrapParams &p = boot.params();
    const Ciphertext in = ev.adjust(x, p.input_level, p.scale);
    if (owned) *owned = Ciphertext();
    const uint32_t unit = members ? members : 1;
    uint32_t step = std::max(unit, batch - batch % unit);
    std::vector<Ciphertext> parts;
    for (uint32_t lo = 0; lo < in.count; lo += step) {
        const uint32_t n = std::min(step, in.count - lo);
        if (members) {
            Ciphertext chunk = ev.slice(in, lo, n);
            const uint32_t pad = (members - n % members) % members;  // a short last group: copies of its first member
            if (pad) chunk = ev.concat(chunk, batch_broadcast(ev, ev.slice(in, lo, 1), pad));
            Ciphertext out = boot.bootstrap_shared_a_s2c_first(chunk, members, &ev);
            parts.push_back(pad ? ev.slice(out, 0, n) : std::move(out));
        } else {
            parts.push_back(boot.bootstrap_ordinary_s2c_first(ev.slice(in, lo, n), &ev));
        }
    }
    return batch_gather(ev, std::move(parts));
}

}  // namespace

Ciphertext bootstrap_segment(const Evaluator &ev, const BatchBootstrapper &boot, const Ciphertext &x,
                             uint32_t members, uint32_t batch) {
    return bootstrap_segment_impl(ev, boot, x, nullptr, members, batch);
}

Ciphertext bootstrap_segment(const Evaluator &ev, const BatchBootstrapper &boot, Ciphertext &&x, uint32_t members,
                             uint32_t batch) {
    return bootstrap_segment_impl(ev, boot, x, &x, members, batch);
}

namespace {

Ciphertext bert_layer_stages(const Evaluator &ev, const BatchBootstrapper &boot, const Ciphertext &X,
                             const BertLayerWeights &w, const BertLayerConfig &cfg, const std::vector<int> &bias_vec,
                             std::vector<StageTime> *times, KeyGenerator *attention_keys, int &stage_no);

const char *const kStageNames[] = {"Attention Block", "SelfOutput", "1st Bootstrapping", "LayerNorm1",
                                   "2nd Bootstrapping", "Intermediate Linear / GELU", "Intermediate Linear / GELU",
                                   "Final Linear", "3rd Bootstrapping", "LayerNorm2", "4th Bootstrapping"};

}  // namespace

Ciphertext bert_layer(const Evaluator &ev, const BatchBootstrapper &boot, const Ciphertext &X,
                      const BertLayerWeights &w, const BertLayerConfig &cfg, const std::vector<int> &bias_vec,
                      std::vector<StageTime> *times, KeyGenerator *attention_keys) {
    int stage_no = 0;
    std::vector<StageTime> local;
    std::vector<StageTime> *tv = times ? times : &local;
    const size_t done0 = tv->size();
    try {
        return bert_layer_stages(ev, boot, X, w, cfg, bias_vec, tv, attention_keys, stage_no);
    } catch (const Error &e) {
        // which stage failed (an allocation failure names only its call site), the device memory in
        // use then and the high-water mark of every finished stage
        std::string msg = std::string(e.what()) + " [bert_layer, stage " + kStageNames[std::min(stage_no, 10)];
        size_t used = 0, reserved = 0;
        if (shm_pool_usage(ev.context().handle(), &reserved, &used, nullptr, 0) == 0) {
            char buf[96];
            std::snprintf(buf, sizeof buf, "; pool %.2f GB used, %.2f GB reserved", used / 1e9, reserved / 1e9);
            msg += buf;
        }
        for (size_t i = done0; i < tv->size(); i++) {
            char buf[128];
            std::snprintf(buf, sizeof buf, "; %s peak %.2f GB", (*tv)[i].name.c_str(), (*tv)[i].peak_bytes / 1e9);
            msg += buf;
        }
        throw Error(msg + "]", e.code);
    }
}

namespace {

Ciphertext bert_layer_stages(const Evaluator &ev, const BatchBootstrapper &boot, const Ciphertext &X,
                             const BertLayerWeights &w, const BertLayerConfig &cfg, const std::vector<int> &bias_vec,
                             std::vector<StageTime> *times, KeyGenerator *attention_keys, int &stage_no) {
    const Context &c = ev.context();
    const uint32_t d = cfg.hidden, H = cfg.heads, dh = d / H, F = cfg.ffn, slots = c.n / 2;
    const uint32_t nb = slots / cfg.tokens;
    if (!H || d % H || X.count != d || X.shared || X.size != 2) throw Error("bert_layer: X must be hidden columns");
    if (cfg.tokens * cfg.num_X != slots) throw Error("bert_layer: num_X * tokens must fill the slots");
    if (bias_vec.size() != slots) throw Error("bert_layer: bias_vec needs one entry per slot");
    auto check_w = [](const std::vector<double> &v, size_t n, const char *what) {
        if (v.size() != n) throw Error(std::string("bert_layer: ") + what + " has the wrong size");
    };
    check_w(w.Wq, (size_t)d * d, "Wq");
    check_w(w.Wk, (size_t)d * d, "Wk");
    check_w(w.Wv, (size_t)d * d, "Wv");
    check_w(w.Wo, (size_t)d * d, "Wo");
    check_w(w.Wi, (size_t)d * F, "Wi");
    check_w(w.Wf, (size_t)F * d, "Wf");
    for (auto *v : {&w.bq, &w.bk, &w.bv, &w.bo, &w.ln1_gamma, &w.ln1_beta, &w.bf, &w.ln2_gamma, &w.ln2_beta})
        check_w(*v, d, "a bias or LayerNorm vector");
    check_w(w.bi, F, "bi");
    const uint32_t top = X.L;
    const double ws = cfg.w_scale;
    double t0 = now_s();
    auto pool_peak = [&](bool reset) {
        size_t high = 0;
        c.check(shm_pool_usage(c.handle(), nullptr, nullptr, &high, reset ? 1 : 0));
        return high;
    };
    pool_peak(true);
    auto stage = [&](const char *name) {
        ev.release_workspace();  // each stage's scratch peak is its own, not the largest so far
        c.synchronize();
        const double t1 = now_s();
        if (times) times->push_back(StageTime{name, t1 - t0, pool_peak(true)});
        t0 = t1;
        stage_no++;
    };

    // ---- Attention Block: per head QKV (one contraction of 3 * dh outputs), QK^T, softmax
    // numerators and their sum; the heads' sums bootstrapped as one batch; inverse, products, * V.
    // With attention_keys the rotation keys of the attention (127 at full width, ~36 GB) are made
    // here and released after it, so they never sit beside the bootstrap and LayerNorm working sets.
    std::map<uint32_t, DeviceBuffer> att_keys;
    Evaluator att_ev(c, ev.encoder());
    att_ev.relin_key = ev.relin_key;
    att_ev.shared_keys = ev.shared_keys;
    att_ev.galois_keys = ev.galois_keys;
    if (attention_keys) {
        // the diagonal packing's baby and giant steps (about 3 sqrt(tokens) of them) stay for the
        // block; the column packing makes its 127 keys a chunk at a time
        uint32_t g = (uint32_t)std::sqrt((double)cfg.tokens);
        if (g * g < cfg.tokens) g++;
        const uint32_t bsteps = (cfg.tokens + g - 1) / g;
        std::set<int> need;
        for (uint32_t j = 1; j < g; j++) need.insert((int)((j * nb) % slots));
        for (uint32_t i = 1; i < bsteps; i++) {
            need.insert((int)(((cfg.tokens - i * g) * nb) % slots));
            need.insert((int)((i * g * nb) % slots));
        }
        for (int st : need)
            if (st) {
                const uint32_t e = ev.galois_elt(st);
                if (!att_keys.count(e)) att_keys.emplace(e, attention_keys->galois_key(e));
            }
        att_ev.galois_keys = &att_keys;
    }
    const Evaluator &aev = attention_keys ? att_ev : ev;
    const double qk_factor = 1.0 / std::sqrt((double)dh);  // the 1/sqrt(d_head) of the scores, in W_q and b_q
    // the inverse of the softmax sum comes back from the bootstrap at X's level less iter + 1:
    // numerators and V wait at that level (products happen there anyway)
    const uint32_t l_inv = top > (uint32_t)cfg.softmax_iter + 2 ? top - (uint32_t)cfg.softmax_iter - 1 : 1;
    std::vector<Ciphertext> numer(H), vals(H), sums(H);
    for (uint32_t h = 0; h < H; h++) {
        std::vector<int64_t> Wqkv((size_t)d * 3 * dh);
        const std::vector<int64_t> q = int_weights(w.Wq, d, d, h * dh, dh, ws, qk_factor),
                                   k = int_weights(w.Wk, d, d, h * dh, dh, ws), v = int_weights(w.Wv, d, d, h * dh, dh, ws);
        for (uint32_t r = 0; r < d; r++) {
            std::copy(q.begin() + (size_t)r * dh, q.begin() + (size_t)(r + 1) * dh, Wqkv.begin() + (size_t)r * 3 * dh);
            std::copy(k.begin() + (size_t)r * dh, k.begin() + (size_t)(r + 1) * dh, Wqkv.begin() + (size_t)r * 3 * dh + dh);
            std::copy(v.begin() + (size_t)r * dh, v.begin() + (size_t)(r + 1) * dh,
                      Wqkv.begin() + (size_t)r * 3 * dh + 2 * dh);
        }
        std::vector<double> b(3 * dh);
        for (uint32_t j = 0; j < dh; j++) {
            b[j] = w.bq[h * dh + j] * qk_factor;
            b[dh + j] = w.bk[h * dh + j];
            b[2 * dh + j] = w.bv[h * dh + j];
        }
        const Ciphertext qkv = add_column_bias(ev, ev.ctpt_matmul(X, Wqkv, 3 * dh, ws), b, bias_vec);
        const Ciphertext S = ct_ct_matmul_colpacking(aev, ev.slice(qkv, 0, dh), ev.slice(qkv, dh, dh), cfg.tokens, nb,
                                                     attention_keys);
        // full rows (every token valid): each cyclic diagonal entry is a valid (query, key) pair, so
        // every slot takes the shift; the reference's band masks assume input_num <= tokens / 2
        numer[h] = cfg.input_num >= cfg.tokens ? exp_approx(ev, ev.add_const(S, kSoftmaxShift))
                                               : softmax_attention_numerators(ev, S, bias_vec, (int)cfg.input_num);
        sums[h] = batch_sum(ev, numer[h]);
        numer[h] = ev.mod_switch_to(numer[h], std::min(numer[h].L, l_inv));
        vals[h] = ev.mod_switch_to(ev.slice(qkv, 2 * dh, dh), numer[h].L);
    }
    const Ciphertext sum_all = bootstrap_segment(ev, boot, batch_gather(ev, sums), cfg.members, cfg.boot_batch);
    const Ciphertext inv_all = inverse_approx(ev, sum_all, cfg.softmax_iter);
    std::vector<Ciphertext> heads(H);
    for (uint32_t h = 0; h < H; h++) {
        const Ciphertext inv = ev.slice(inv_all, h, 1);
        const Ciphertext sm = ev.relinearize_rescale(ev.multiply_lazy(numer[h], batch_broadcast(ev, inv, numer[h].count)));
        numer[h] = Ciphertext();
        heads[h] = ct_ct_matmul_diagpacking(aev, sm, ev.mod_switch_to(vals[h], sm.L), nb);
        vals[h] = Ciphertext();
    }
    Ciphertext att = batch_gather(ev, std::move(heads));
    heads.clear();
    att_keys.clear();
    att_ev.release_workspace();
    stage("Attention Block");

    // ---- SelfOutput
    Ciphertext so = add_column_bias(ev, ev.ctpt_matmul(att, int_weights(w.Wo, d, d, 0, d, ws), d, ws), w.bo, bias_vec);
    att = Ciphertext();
    stage("SelfOutput");
    Ciphertext b1 = bootstrap_segment(ev, boot, std::move(so), cfg.members, cfg.boot_batch);
    stage("1st Bootstrapping");

    // ---- LayerNorm1 on SelfOutput + X
    Ciphertext res1 = ev.add(b1, ev.mod_switch_to(X, b1.L));
    b1 = Ciphertext();
    Ciphertext ln1 = layernorm(ev, std::move(res1), w.ln1_gamma, w.ln1_beta, cfg.ln_newt, cfg.ln_gold,
                               cfg.ln_var_scale);
    stage("LayerNorm1");
    Ciphertext H1 = bootstrap_segment(ev, boot, std::move(ln1), cfg.members, cfg.boot_batch);
    stage("2nd Bootstrapping");

    // ---- Intermediate + GELU in column chunks (each chunk's GELU working set stays bounded)
    const uint32_t l_inter = std::min(H1.L, cfg.gelu_input_level + 1);
    Ciphertext h1i = ev.mod_switch_to(H1, l_inter);
    std::vector<Ciphertext> g;
    double t_inter = 0, t_gelu = 0;
    for (uint32_t lo = 0; lo < F; lo += cfg.ffn_chunk) {
        const uint32_t n = std::min(cfg.ffn_chunk, F - lo);
        double ta = now_s();
        const std::vector<double> bi(w.bi.begin() + lo, w.bi.begin() + lo + n);
        const Ciphertext I = add_column_bias(ev, ev.ctpt_matmul(h1i, int_weights(w.Wi, d, F, lo, n, ws), n, ws), bi,
                                             bias_vec);
        c.synchronize();
        double tb = now_s();
        g.push_back(gelu(ev, I));
        c.synchronize();
        t_inter += tb - ta;
        t_gelu += now_s() - tb;
    }
    h1i = Ciphertext();
    if (times) {
        const size_t high = pool_peak(true);
        times->push_back(StageTime{"Intermediate Linear", t_inter, high});
        times->push_back(StageTime{"GELU", t_gelu, high});
    }
    stage_no += 2;
    t0 = now_s();

    // ---- Final (masked by bias_vec: the padding slots GELU left non-zero are cleared)
    Ciphertext G = batch_gather(ev, std::move(g));
    std::vector<double> mask(bias_vec.begin(), bias_vec.end());
    Ciphertext fin = add_column_bias(ev, ev.ctpt_matmul_masked(G, int_weights(w.Wf, F, d, 0, d, ws), d, ws, mask),
                                     w.bf, bias_vec);
    G = Ciphertext();
    stage("Final Linear");
    Ciphertext b3 = bootstrap_segment(ev, boot, std::move(fin), cfg.members, cfg.boot_batch);
    stage("3rd Bootstrapping");

    // ---- LayerNorm2 on Final + H1
    Ciphertext res2 = ev.add(b3, ev.mod_switch_to(H1, b3.L));
    b3 = Ciphertext();
    H1 = Ciphertext();
    Ciphertext ln2 = layernorm(ev, std::move(res2), w.ln2_gamma, w.ln2_beta, cfg.ln_newt, cfg.ln_gold,
                               cfg.ln_var_scale);
    stage("LayerNorm2");
    Ciphertext out = bootstrap_segment(ev, boot, std::move(ln2), cfg.members, cfg.boot_batch);
    stage("4th Bootstrapping");
    (void)top;
    return out;
}

}  // namespace

}  // namespace shmoai
