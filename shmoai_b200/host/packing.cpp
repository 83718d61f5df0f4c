// The MOAI driver's packing of a batch of inputs into ciphertexts
// (src/include/source/matrix_mul/Batch_encode_encrypt.cuh): the column-interleaved
// layout every BERT-layer operator works on, and its valid-slot mask.
#include "internal.hpp"

namespace shmoai {

Ciphertext batch_input(PublicEncryptor &enc, const std::vector<double> &X, uint32_t num_X, uint32_t num_row,
                       uint32_t num_col, double scale, uint32_t L) {
    const size_t per = (size_t)num_row * num_col;
    if (!num_X || !num_row || !num_col) throw Error("batch_input: empty batch");
    if (X.size() != (size_t)num_X * per) throw Error("batch_input: X must hold num_X * num_row * num_col values");
    // one slot vector per column; the trailing zero slots are left to the encoder's padding
    std::vector<std::vector<cplx>> z(num_col, std::vector<cplx>((size_t)num_X * num_row));
    for (uint32_t j = 0; j < num_X; j++)
        for (uint32_t k = 0; k < num_row; k++) {
            const double *row = X.data() + (size_t)j * per + (size_t)k * num_col;
            for (uint32_t i = 0; i < num_col; i++) z[i][(size_t)num_X * k + j] = cplx(row[i], 0.0);
        }
    return enc.encrypt(z, scale, L);
}

std::vector<int> bias_vec(const std::vector<int> &lengths, uint32_t num_X, uint32_t num_row) {
    if (lengths.size() != num_X) throw Error("bias_vec: one length per input");
    std::vector<int> out((size_t)num_X * num_row, 0);
    for (uint32_t i = 0; i < num_X; i++) {
        if (lengths[i] < 0 || (uint32_t)lengths[i] > num_row) throw Error("bias_vec: length out of range");
        for (int j = 0; j < lengths[i]; j++) out[(size_t)j * num_X + i] = 1;
    }
    return out;
}

}  // namespace shmoai
