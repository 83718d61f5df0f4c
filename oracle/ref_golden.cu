// Golden-vector generator: runs the REFERENCE evaluator (ShMOAI's PhantomFHE
// plus its moai:: adapter, built for sm_100a from the reference sources by
// oracle/build_ref.sh) on deterministic inputs and prints a JSON record of
// every output (checksum + first coefficients of each limb).
//
// TEST INFRASTRUCTURE ONLY.  Inputs and key material are not sampled by the
// reference: they are filled from the counter generator below, which the
// Python tests regenerate bit for bit, so no large arrays have to be stored.
//
//   usage: ref_golden <tiny|prim|boot> > golden.json
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "phantom.h"
#include "ckks_evaluator_parallel.cuh"

using namespace phantom;
using namespace phantom::arith;
using namespace phantom::util;

static uint64_t sm64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// value of flat element e of a tagged array whose row r (length n) lives under prime primes[row_prime[r]]
static void fill(std::vector<uint64_t> &v, uint64_t tag, size_t n, const std::vector<uint64_t> &row_mod) {
    for (size_t e = 0; e < v.size(); e++) v[e] = sm64((tag << 40) + e) % row_mod[e / n];
}

static uint64_t checksum(const std::vector<uint64_t> &v) {
    uint64_t h = 0;
    for (size_t e = 0; e < v.size(); e++) h += sm64(v[e] ^ (e * 0x9E3779B97F4A7C15ull));
    return h;
}

static std::vector<uint64_t> d2h(const uint64_t *p, size_t count) {
    std::vector<uint64_t> v(count);
    cudaDeviceSynchronize();
    cudaMemcpy(v.data(), p, count * sizeof(uint64_t), cudaMemcpyDeviceToHost);
    return v;
}

static void h2d(uint64_t *p, const std::vector<uint64_t> &v) {
    cudaDeviceSynchronize();
    cudaMemcpy(p, v.data(), v.size() * sizeof(uint64_t), cudaMemcpyHostToDevice);
    cudaDeviceSynchronize();
}

static bool first_record = true;
static void emit(const char *name, const std::vector<uint64_t> &v, size_t rows, size_t n, const char *extra = "") {
    printf("%s\n  \"%s\": {\"rows\": %zu, \"n\": %zu, \"checksum\": \"%016llx\"%s, \"head\": [", first_record ? "" : ",",
           name, rows, n, (unsigned long long)checksum(v), extra);
    first_record = false;
    for (size_t r = 0; r < rows; r++) {
        printf("%s[", r ? ", " : "");
        for (size_t k = 0; k < 8; k++) printf("%s\"%llu\"", k ? ", " : "", (unsigned long long)v[r * n + k]);
        printf("]");
    }
    printf("]}");
}

static double weight(uint64_t tag, uint64_t i) {
    // exactly reproducible in numpy: a 53-bit integer times a constant
    int64_t m = (int64_t)(sm64((tag << 40) + i) >> 11) - (int64_t(1) << 52);
    return (double)m * (0.08 / 4503599627370496.0);
}

int main(int argc, char **argv) {
    std::string which = argc > 1 ? argv[1] : "tiny";
    int log_n;
    std::vector<int> bits;
    size_t np;
    if (which == "tiny") {
        log_n = 12;
        bits = {60, 50, 50, 50, 50, 50, 60, 60};
        np = 2;
    } else if (which == "prim") {
        log_n = 16;
        bits.push_back(60);
        for (int i = 0; i < 23; i++) bits.push_back(50);
        for (int i = 0; i < 8; i++) bits.push_back(60);
        np = 8;
    } else {
        log_n = 16;
        bits.push_back(51);
        for (int i = 0; i < 20; i++) bits.push_back(46);
        for (int i = 0; i < 14; i++) bits.push_back(51);
        for (int i = 0; i < 5; i++) bits.push_back(51);
        np = 5;
    }
    size_t N = size_t(1) << log_n, QP = bits.size(), nq = QP - np, L = nq, dnum = nq / np;

    EncryptionParameters parms(scheme_type::ckks);
    parms.set_poly_modulus_degree(N);
    parms.set_coeff_modulus(CoeffModulus::Create(N, bits));
    parms.set_special_modulus_size(np);
    PhantomContext context(parms);
    PhantomCKKSEncoder encoder(context);
    moai::Encoder enc(&context, &encoder);
    moai::Evaluator ev(&context, &encoder);
    PhantomSecretKey sk(context);
    PhantomRelinKey rk = sk.gen_relinkey(context);
    PhantomGaloisKey gk = sk.create_galois_keys_from_steps(context, {0, 1});
    const auto &s = global_variables::default_stream->get_stream();

    std::vector<uint64_t> primes(QP);
    for (size_t i = 0; i < QP; i++) primes[i] = parms.coeff_modulus()[i].value();

    printf("{\n  \"params\": {\"name\": \"%s\", \"log_n\": %d, \"nq\": %zu, \"np\": %zu, \"dnum\": %zu, \"primes\": [",
           which.c_str(), log_n, nq, np, dnum);
    for (size_t i = 0; i < QP; i++) printf("%s\"%llu\"", i ? ", " : "", (unsigned long long)primes[i]);
    printf("]}");
    first_record = false;

    // ---- key material: overwrite the reference's keys with generator data
    auto key_rows = [&]() {
        std::vector<uint64_t> rm;
        for (int h = 0; h < 2; h++)
            for (size_t i = 0; i < QP; i++) rm.push_back(primes[i]);
        return rm;
    };
    auto load_key = [&](const PhantomRelinKey &key, uint64_t tag) {
        std::vector<uint64_t *> ptrs(dnum);
        cudaDeviceSynchronize();
        cudaMemcpy(ptrs.data(), key.public_keys_ptr(), dnum * sizeof(uint64_t *), cudaMemcpyDeviceToHost);
        for (size_t d = 0; d < dnum; d++) {
            std::vector<uint64_t> v(2 * QP * N);
            fill(v, tag + d, N, key_rows());
            h2d(ptrs[d], v);
        }
    };
    // tags: relin key 100+d, galois(elt 2N-1) 200+d, galois(elt 5) 300+d
    load_key(rk, 100);
    {
        auto &elts = context.key_galois_tool_->galois_elts();
        for (size_t idx = 0; idx < elts.size(); idx++) load_key(gk.get_relin_keys(idx), elts[idx] == 5 ? 300 : 200);
    }

    std::vector<uint64_t> qrows;
    for (int h = 0; h < 3; h++)
        for (size_t i = 0; i < L; i++) qrows.push_back(primes[i]);

    auto make_ct = [&](uint64_t tag, size_t limbs) {
        PhantomCiphertext ct;
        size_t chain = 1 + (L - limbs);
        ct.resize(context, chain, 2, s);
        ct.set_scale(std::pow(2.0, 40));
        ct.set_ntt_form(true);
        std::vector<uint64_t> rows;
        for (int h = 0; h < 2; h++)
            for (size_t i = 0; i < limbs; i++) rows.push_back(primes[i]);
        std::vector<uint64_t> v(2 * limbs * N);
        fill(v, tag, N, rows);
        h2d(ct.data(), v);
        return ct;
    };
    auto dump_ct = [&](const char *name, const PhantomCiphertext &ct) {
        size_t rows = ct.size() * ct.coeff_modulus_size();
        emit(name, d2h(ct.data(), rows * N), rows, N);
    };

    // inputs: A (tag 1), B (tag 2) at the top level; plaintext C (tag 3)
    PhantomCiphertext A = make_ct(1, L), B = make_ct(2, L);

    {   // NTT both ways (moai adapter, ckks_evaluator_parallel.cuh:396-442)
        PhantomCiphertext t;
        ev.transform_from_ntt(A, t);
        dump_ct("intt_A", t);
        PhantomCiphertext u;
        ev.transform_to_ntt(A, u);
        dump_ct("ntt_A", u);
    }
    {   // element-wise
        PhantomCiphertext t;
        ev.add(A, B, t);
        dump_ct("add_AB", t);
        PhantomPlaintext C;
        C.resize(L, N, s);
        C.set_chain_index(1);
        std::vector<uint64_t> v(L * N);
        fill(v, 3, N, qrows);
        h2d(C.data(), v);
        PhantomCiphertext u;
        ev.multiply_plain(A, C, u);
        dump_ct("mulplain_AC", u);
    }
    {   // rescale (floor)
        PhantomCiphertext t = A;
        ev.rescale_to_next_inplace(t);
        dump_ct("rescale_A", t);
    }
    {   // rotation by one slot and conjugation
        PhantomCiphertext t = A;
        ev.rotate_vector_inplace(t, 1, gk);
        dump_ct("rot1_A", t);
        PhantomCiphertext u;
        ev.complex_conjugate(A, gk, u);
        dump_ct("conj_A", u);
    }
    {   // multiply -> relinearize -> rescale
        PhantomCiphertext t;
        ev.multiply(A, B, t);
        dump_ct("mul_AB", t);
        ev.relinearize_inplace(t, rk);
        dump_ct("relin_AB", t);
        ev.rescale_to_next_inplace(t);
        dump_ct("mrr_AB", t);
    }
    {   // key switching one level down: the last digit is short
        PhantomCiphertext D = make_ct(4, L - 1);
        PhantomCiphertext t = D;
        ev.rotate_vector_inplace(t, 1, gk);
        dump_ct("rot1_D", t);
        PhantomCiphertext E = make_ct(5, L - 1), u;
        ev.multiply(D, E, u);
        ev.relinearize_inplace(u, rk);
        dump_ct("relin_DE", u);
    }
    {   // constant encodes at scale 2^40: coefficient-0 integer via limb 0 of the NTT form
        const size_t K = which == "tiny" ? 2048 : 256;
        printf(",\n  \"encode_w\": {\"scale_log2\": 40, \"values\": [");
        for (size_t i = 0; i < K + 64; i++) {
            double w = i < K ? weight(7, i) : (std::ldexp(double((int64_t)(sm64(i) % 2000000) - 1000000) + 0.5, -40));
            PhantomPlaintext pt;
            enc.encode(w, 1, std::pow(2.0, 40), pt);
            auto v = d2h(pt.data(), L * N);
            bool constant = true;
            for (size_t r = 0; r < L && constant; r++)
                for (size_t k = 1; k < N; k++)
                    if (v[r * N + k] != v[r * N]) { constant = false; break; }
            int64_t c = v[0] > primes[0] / 2 ? -(int64_t)(primes[0] - v[0]) : (int64_t)v[0];
            printf("%s[%.17g, \"%lld\", %d]", i ? ", " : "", w, (long long)c, constant ? 1 : 0);
        }
        printf("]}");
    }
    {   // rotation-free ct-pt matmul, the reference loop (Ct_pt_matrix_mul.cuh:112-158)
        const size_t n_in = 8, n_out = 4;
        std::vector<PhantomCiphertext> X;
        for (size_t j = 0; j < n_in; j++) X.push_back(make_ct(20 + j, L));
        printf(",\n  \"ctpt_w\": [");
        for (size_t j = 0; j < n_in; j++)
            for (size_t o = 0; o < n_out; o++) printf("%s%.17g", j + o ? ", " : "", weight(8, j * n_out + o));
        printf("]");
        for (size_t o = 0; o < n_out; o++) {
            printf(",\n  \"ctpt_wint_%zu\": [", o);
            PhantomCiphertext acc;
            for (size_t j = 0; j < n_in; j++) {
                PhantomPlaintext pt;
                enc.encode(weight(8, j * n_out + o), X[j].chain_index(), X[j].scale(), pt);
                auto v = d2h(pt.data(), N);
                int64_t c = v[0] > primes[0] / 2 ? -(int64_t)(primes[0] - v[0]) : (int64_t)v[0];
                printf("%s\"%lld\"", j ? ", " : "", (long long)c);
                PhantomCiphertext t;
                ev.multiply_plain(X[j], pt, t);
                if (j == 0) acc = t;
                else ev.add_inplace(acc, t);
            }
            char nm[32];
            snprintf(nm, sizeof nm, "ctpt_sum_%zu", o);
            // sums are dumped before the rescale, then the rescaled output
            size_t rows = 2 * L;
            auto sum = d2h(acc.data(), rows * N);
            printf("]");
            emit(nm, sum, rows, N);
            ev.rescale_to_next_inplace(acc);
            snprintf(nm, sizeof nm, "ctpt_out_%zu", o);
            dump_ct(nm, acc);
        }
    }
    printf("\n}\n");
    cudaDeviceSynchronize();
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
