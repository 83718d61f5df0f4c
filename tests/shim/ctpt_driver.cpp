// The reference's config-2 driver (src/include/test/matrix_mul/test_ct_pt_matrix_mul.cuh:7-169)
// restated over the moai / PhantomFHE names that include/moai_shim.hpp provides: parameters,
// keys, the column-interleaved batch of inputs X_i[j][k] = j + 1, the all-1/128 weight matrix,
// ct_pt_matrix_mul_wo_pre, then decrypt + decode of every output against the closed form
// (j + 1) * num_col / 128 on the slots of token j.  Sizes come from the command line so the CPU
// test runs a reduced case: log_n num_X num_row num_col col_W.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "moai_shim.hpp"

using namespace std;
using namespace phantom;
using namespace moai;

int main(int argc, char **argv) {
    const int log_n = argc > 1 ? atoi(argv[1]) : 16;
    const int num_X = argc > 2 ? atoi(argv[2]) : 256;
    const int num_row = argc > 3 ? atoi(argv[3]) : 128;
    const int num_col = argc > 4 ? atoi(argv[4]) : 768;
    const int col_W = argc > 5 ? atoi(argv[5]) : 64;

    EncryptionParameters parms(scheme_type::ckks);
    size_t poly_modulus_degree = size_t(1) << log_n;
    parms.set_poly_modulus_degree(poly_modulus_degree);
    parms.set_coeff_modulus(CoeffModulus::Create(poly_modulus_degree,
                                                 {60, 40, 40, 40, 40, 40, 40, 40, 40, 40, 40, 40, 40, 40, 40, 60}));
    parms.set_sparse_slots(poly_modulus_degree / 2);
    double scale = pow(2.0, 40);
    PhantomContext context(parms);

    PhantomSecretKey secret_key(context);
    PhantomPublicKey public_key = secret_key.gen_publickey(context);
    Decryptor decryptor(&context, &secret_key);
    PhantomCKKSEncoder phantom_encoder(context);
    Encoder encoder(&context, &phantom_encoder);
    Encryptor encryptor(&context, &public_key);
    Evaluator evaluator(&context, &phantom_encoder);
    size_t slot_count = encoder.slot_count();

    vector<vector<vector<double>>> input_x(num_X, vector<vector<double>>(num_row, vector<double>(num_col, 0)));
    for (int i = 0; i < num_X; ++i)
        for (int j = 0; j < num_row; ++j)
            for (int k = 0; k < num_col; ++k) input_x[i][j][k] = (double)j + 1.0;
    vector<PhantomCiphertext> enc_ecd_x = batch_input(input_x, num_X, num_row, num_col, scale, context, public_key);

    vector<vector<double>> W(num_col, vector<double>(col_W, 1.0 / 128.0));
    vector<PhantomCiphertext> ct_pt_mul = ct_pt_matrix_mul_wo_pre(enc_ecd_x, W, num_col, col_W, num_col, context);

    double max_err = 0;
    for (int i = 0; i < col_W; ++i) {
        PhantomPlaintext plain_result;
        decryptor.decrypt(ct_pt_mul[i], plain_result);
        vector<double> result;
        encoder.decode(plain_result, result);
        for (size_t ind = 0; ind < slot_count; ++ind) {
            const int j = (int)(ind / num_X);  // token row of slot num_X * j + input
            const double want = j < num_row ? (j + 1.0) * num_col / 128.0 : 0.0;
            max_err = fmax(max_err, fabs(result[ind] - want) / fmax(1.0, fabs(want)));
        }
    }
    printf("outputs %d chain_index %zu coeff_modulus_size %zu scale_log2 %.3f max_rel_err %.3e\n", col_W,
           ct_pt_mul[0].chain_index(), ct_pt_mul[0].coeff_modulus_size(), log2(ct_pt_mul[0].scale()), max_err);
    return max_err < 1e-5 ? 0 : 1;
}
