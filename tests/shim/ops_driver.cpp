// MOAI-style calls through include/moai_shim.hpp on one ciphertext: encode / encrypt with the
// public key, multiply + relinearize_inplace + rescale_to_next_inplace, rotate_vector_inplace,
// complex_conjugate, multiply_const + rescale, PhantomCKKSEncoder::encode at a chain index +
// add_plain_inplace, mod_switch_to_next_inplace; every result decrypted and decoded against the
// slot arithmetic.
// Argument: log_n.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "moai_shim.hpp"

using namespace std;
using namespace phantom;
using namespace moai;

static double worst = 0;

static void check(const char *what, const vector<complex<double>> &got, const vector<complex<double>> &want,
                  double tol) {
    double e = 0;
    for (size_t i = 0; i < want.size(); i++) e = fmax(e, abs(got[i] - want[i]));
    printf("%-18s max_err %.3e\n", what, e);
    if (!(e < tol)) worst = 1;
}

int main(int argc, char **argv) {
    const int log_n = argc > 1 ? atoi(argv[1]) : 12;
    const size_t N = size_t(1) << log_n;
    EncryptionParameters parms(scheme_type::ckks);
    parms.set_poly_modulus_degree(N);
    parms.set_coeff_modulus(CoeffModulus::Create(N, {60, 40, 40, 40, 40, 40, 60, 60}));
    parms.set_special_modulus_size(2);
    PhantomContext context(parms);
    PhantomSecretKey sk(context, 64, 17);
    PhantomPublicKey pk = sk.gen_publickey(context);
    PhantomRelinKey rk = sk.gen_relinkey(context);
    PhantomGaloisKey gk = sk.create_galois_keys_from_steps(context, {0, 1, -3});
    PhantomCKKSEncoder penc(context);
    Encoder encoder(&context, &penc);
    Encryptor encryptor(&context, &pk);
    Decryptor decryptor(&context, &sk);
    Evaluator evaluator(&context, &penc);
    const double scale = pow(2.0, 40);
    const size_t slots = encoder.slot_count();

    vector<complex<double>> x(slots), y(slots);
    for (size_t i = 0; i < slots; i++) {
        x[i] = complex<double>(sin(0.01 * i), cos(0.03 * i)) * 0.8;
        y[i] = complex<double>(cos(0.02 * i), 0.5 * sin(0.05 * i)) * 0.8;
    }
    auto enc = [&](const vector<complex<double>> &v) {
        PhantomPlaintext p;
        encoder.encode(v, scale, p);
        PhantomCiphertext c;
        encryptor.encrypt(p, c);
        return c;
    };
    auto dec = [&](PhantomCiphertext &c) {
        PhantomPlaintext p;
        decryptor.decrypt(c, p);
        vector<complex<double>> v;
        encoder.decode(p, v);
        return v;
    };
    PhantomCiphertext cx = enc(x), cy = enc(y);
    check("encrypt", dec(cx), x, 1e-6);

    PhantomCiphertext m;
    evaluator.multiply(cx, cy, m);
    evaluator.relinearize_inplace(m, rk);
    evaluator.rescale_to_next_inplace(m);
    vector<complex<double>> xy(slots);
    for (size_t i = 0; i < slots; i++) xy[i] = x[i] * y[i];
    check("mul_relin_rescale", dec(m), xy, 1e-5);

    PhantomCiphertext r = cx;
    evaluator.rotate_vector_inplace(r, 1, gk);
    vector<complex<double>> rx(slots);
    for (size_t i = 0; i < slots; i++) rx[i] = x[(i + 1) % slots];
    check("rotate 1", dec(r), rx, 1e-5);
    evaluator.rotate_vector_inplace(r, -3, gk);
    for (size_t i = 0; i < slots; i++) rx[i] = x[(i + slots - 2) % slots];
    check("rotate 1 - 3", dec(r), rx, 1e-5);

    PhantomCiphertext cc;
    evaluator.complex_conjugate(cx, gk, cc);
    vector<complex<double>> cj(slots);
    for (size_t i = 0; i < slots; i++) cj[i] = conj(x[i]);
    check("conjugate", dec(cc), cj, 1e-5);

    PhantomCiphertext k;
    evaluator.multiply_const(cx, 0.375, k);
    evaluator.rescale_to_next_inplace(k);
    PhantomPlaintext py;
    penc.encode(context, y, k.scale(), py, k.chain_index());
    evaluator.add_plain_inplace(k, py);
    vector<complex<double>> ax(slots);
    for (size_t i = 0; i < slots; i++) ax[i] = 0.375 * x[i] + y[i];
    check("const + add_plain", dec(k), ax, 1e-5);

    PhantomCiphertext d = cx;
    evaluator.mod_switch_to_next_inplace(d);
    if (d.coeff_modulus_size() + 1 != cx.coeff_modulus_size() || d.chain_index() != cx.chain_index() + 1) worst = 1;
    check("mod_switch", dec(d), x, 1e-6);

    printf("%s\n", worst ? "FAIL" : "ok");
    return worst ? 1 : 0;
}
