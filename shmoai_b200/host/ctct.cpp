// Ciphertext-ciphertext matrix products of the attention block.  Column packing
// (ct_ct_matrix_mul_colpacking, src/include/source/matrix_mul/Ct_ct_matrix_mul.cuh:10-120):
// out_i = sum_j X_j * rot(W_j, i * num_batch), one relinearisation and rescale per output.
// The rotations of W are hoisted (one ModUp of the whole W batch for every step) and the
// products are summed unrelinearised (size 3) in one pass, as the reference sums before
// relinearising.
#include <algorithm>
#include <cmath>

#include "internal.hpp"

namespace shmoai {

Ciphertext ct_ct_matmul_colpacking(const Evaluator &ev, const Ciphertext &X, const Ciphertext &W, uint32_t rows,
                                   uint32_t num_batch, KeyGenerator *keys) {
    if (X.shared || W.shared || X.size != 2 || W.size != 2) throw Error("ct-ct matmul takes ordinary ciphertexts");
    if (X.count != W.count || X.count == 0) throw Error("ct-ct matmul: X and W need the same number of columns");
    if (rows == 0) throw Error("ct-ct matmul: no output rows");
    // the rotated copies of W are made a chunk of steps at a time (one hoisted ModUp per chunk), so
    // at most ~12 GB of them are live: at full width a head's 127 rotations of 64 ciphertexts would
    // otherwise hold 170 GB
    // With `keys`, the Galois keys of a chunk's steps are made for that chunk and released after
    // it (at full width the 127 keys would hold ~36 GB for the whole product).
    const size_t w_bytes = W.polys() * W.L * ev.context().n * 8;
    const uint32_t chunk = (uint32_t)std::max<size_t>(1, (size_t(12) << 30) / std::max<size_t>(w_bytes, 1));
    std::vector<Ciphertext> outs;
    outs.reserve(rows);
    for (uint32_t lo = 0; lo < rows; lo += chunk) {
        const uint32_t hi = std::min(rows, lo + chunk);
        std::vector<int> steps;
        for (uint32_t i = std::max(lo, 1u); i < hi; i++) steps.push_back((int)(i * num_batch));
        std::map<uint32_t, DeviceBuffer> chunk_keys;
        Evaluator kev(ev.context(), ev.encoder());
        kev.relin_key = ev.relin_key;
        kev.galois_keys = &chunk_keys;
        if (keys)
            for (int st : steps) {
                const uint32_t e = ev.galois_elt(st);
                if (!chunk_keys.count(e)) chunk_keys.emplace(e, keys->galois_key(e));
            }
        const std::map<int, Ciphertext> rot = (keys ? kev : ev).rotate_many(W, steps);
        // each row's products summed in one pass (no size-3 batch of the products), and the chunk's
        // rows relinearised and rescaled as one batch
        std::vector<Ciphertext> sums;
        for (uint32_t i = lo; i < hi; i++) {
            const int step = (int)(i * num_batch);
            auto it = rot.find(step);
            const Ciphertext &Wi = (i == 0 || it == rot.end()) ? W : it->second;  // a full turn is W itself
            sums.push_back(ev.sum_of_products(X, Wi));
        }
        outs.push_back(ev.relinearize_rescale(batch_gather(ev, std::move(sums))));
    }
    return batch_gather(ev, std::move(outs));
}

Ciphertext ct_ct_matmul_diagpacking(const Evaluator &ev, const Ciphertext &X, const Ciphertext &W,
                                    uint32_t num_batch) {
    if (X.shared || W.shared || X.size != 2 || W.size != 2) throw Error("ct-ct matmul takes ordinary ciphertexts");
    const uint32_t col = X.count, cw = W.count;
    if (col == 0 || cw == 0) throw Error("ct-ct matmul: empty batch");
    const int64_t slots = ev.context().n / 2;
    auto norm = [&](int64_t k) { return (int)(((k % slots) + slots) % slots); };
    uint32_t g = (uint32_t)std::sqrt((double)col);
    if (g * g < col) g++;
    uint32_t b = col / g;
    if (b * g < col) b++;
    // giant-step groups of X: members i g .. i g + g - 1 rotated by (col - i g) num_batch
    std::vector<Ciphertext> rx;  // one batch per giant step
    for (uint32_t i = 0; i < b; i++) {
        const uint32_t lo = i * g, cnt = std::min(g, col - lo);
        Ciphertext grp = ev.slice(X, lo, cnt);
        const int step = norm((int64_t)(col - i * g) * num_batch);
        if (i == 0 || step == 0) {
            rx.push_back(std::move(grp));
        } else {
            auto r = ev.rotate_many(grp, {step});
            rx.push_back(std::move(r.at(step)));
        }
    }
    // baby steps of W: rot(W, j num_batch), j < g, hoisted over the whole W batch
    std::vector<int> bsteps;
    for (uint32_t j = 1; j < g; j++) bsteps.push_back(norm((int64_t)j * num_batch));
    const std::map<int, Ciphertext> wr = ev.rotate_many(W, bsteps);
    auto baby = [&](uint32_t j) -> const Ciphertext & {
        const int st = j ? norm((int64_t)j * num_batch) : 0;
        auto it = wr.find(st);
        return (j == 0 || it == wr.end()) ? W : it->second;
    };
    Ciphertext total;
    for (uint32_t i = 0; i < b; i++) {
        // sum_k baby(k) x X's member k of the group, X's member broadcast over W's batch, summed in one pass
        std::vector<Ciphertext> xs;
        std::vector<const Ciphertext *> As, Bs;
        for (uint32_t k = 0; k < g && i * g + k < col; k++) xs.push_back(ev.slice(rx[i], k, 1));
        for (uint32_t k = 0; k < xs.size(); k++) {
            As.push_back(&baby(k));
            Bs.push_back(&xs[k]);
        }
        Ciphertext o = ev.relinearize_rescale(ev.multiply_accumulate(As, Bs));
        const int gs = norm((int64_t)i * g * num_batch);
        if (i > 0 && gs != 0) o = std::move(ev.rotate_many(o, {gs}).at(gs));
        total = total.count ? ev.add(total, o) : std::move(o);
    }
    return total;
}

}  // namespace shmoai
