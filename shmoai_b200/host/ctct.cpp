// Ciphertext-ciphertext matrix product of the attention block in the column packing
// (ct_ct_matrix_mul_colpacking, src/include/source/matrix_mul/Ct_ct_matrix_mul.cuh:10-120):
// out_i = sum_j X_j * rot(W_j, i * num_batch), one relinearisation and rescale per output.
// The rotations of W are hoisted (one ModUp of the whole W batch for every step) and the
// products are summed unrelinearised (size 3), as the reference sums before relinearising.
#include "internal.hpp"

namespace shmoai {

namespace {

// sum over a batch of ordinary ciphertexts of any size (2 or 3): halves added pairwise
Ciphertext sum_members(const Evaluator &ev, Ciphertext cur) {
    while (cur.count > 1) {
        const uint32_t h = cur.count / 2;
        Ciphertext s = ev.add(ev.slice(cur, 0, h), ev.slice(cur, h, h));
        if (cur.count & 1) s = ev.concat(s, ev.slice(cur, 2 * h, 1));
        cur = std::move(s);
    }
    return cur;
}

}  // namespace

Ciphertext ct_ct_matmul_colpacking(const Evaluator &ev, const Ciphertext &X, const Ciphertext &W, uint32_t rows,
                                   uint32_t num_batch) {
    if (X.shared || W.shared || X.size != 2 || W.size != 2) throw Error("ct-ct matmul takes ordinary ciphertexts");
    if (X.count != W.count || X.count == 0) throw Error("ct-ct matmul: X and W need the same number of columns");
    if (rows == 0) throw Error("ct-ct matmul: no output rows");
    std::vector<int> steps;
    for (uint32_t i = 1; i < rows; i++) steps.push_back((int)(i * num_batch));
    const std::map<int, Ciphertext> rot = ev.rotate_many(W, steps);
    std::vector<Ciphertext> outs;
    outs.reserve(rows);
    for (uint32_t i = 0; i < rows; i++) {
        const int step = (int)(i * num_batch);
        auto it = rot.find(step);
        const Ciphertext &Wi = (i == 0 || it == rot.end()) ? W : it->second;  // a full turn is W itself
        outs.push_back(ev.relinearize_rescale(sum_members(ev, ev.multiply_lazy(X, Wi))));
    }
    return batch_gather(ev, outs);
}

}  // namespace shmoai
