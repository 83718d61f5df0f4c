// The softmax's building blocks on ciphertext batches (src/include/source/non_linear_func/
// softmax.cuh:23-118): exp by (1 + x/128)^128 and 1/x by the product prod_i (1 + y^(2^i)),
// y = 1 - x.  Products are relinearised and rescaled in one ModDown (relinearize_rescale).
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
    if (x.L < 10) throw Error("exp needs 8 levels and one prime for its output");
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

}  // namespace shmoai
