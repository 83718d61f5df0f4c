// Golden-vector generator: runs the REFERENCE evaluator (ShMOAI's PhantomFHE
// plus its moai:: adapter, built for sm_100a from the reference sources by
// oracle/build_ref.sh) on deterministic inputs and prints a JSON record of
// every output (checksum + first coefficients of each limb).
//
// TEST INFRASTRUCTURE ONLY.  Inputs and key material are not sampled by the
// reference: they are filled from the counter generator below, which the
// Python tests regenerate bit for bit, so no large arrays have to be stored.
//
//   usage: ref_golden <tiny|prim|boot> [golden|shared|time] > out.json
//
//   golden  the evaluator records (NTT, add, multiply_plain, rescale, rotate,
//           conjugate, multiply, relinearize, constant encodes, ct-pt loop)
//   shared  the shared-a records (FmtSwitch forward / backward, Sh-Rot, the
//           shared batch rescale / modraise / multiply_plain / add) and a
//           complex slot-vector encode; params.name is "shared_<set>"
//   time    CUDA-event timings of the reference's own calls on this GPU (the
//           config-1 primitives, per-ciphertext HRotate and multiply +
//           relinearize + rescale, the per-ciphertext ct-pt loop)
#include <omp.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "phantom.h"
#include "ckks_evaluator_parallel.cuh"
#include "FmtSwitch.cuh"
#include "ShRotate.cuh"
#include "SharedABatchOps.cuh"

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

// slot value in [-1, 1): a 53-bit integer times 2^-52 minus one, exactly reproducible in numpy
static double unit(uint64_t tag, uint64_t i) {
    return (double)(sm64((tag << 40) + i) >> 11) * (1.0 / 4503599627370496.0) - 1.0;
}

struct Env {
    PhantomContext &context;
    PhantomCKKSEncoder &encoder;
    moai::Encoder &enc;
    moai::Evaluator &ev;
    PhantomSecretKey &sk;
    PhantomRelinKey &rk;
    PhantomGaloisKey &gk;
    std::vector<uint64_t> primes;
    size_t N, nq, np, dnum, QP;
    int log_n;
    cudaStream_t s;
};

// rows of a tag-filled array: `reps` copies of the given prime list
static std::vector<uint64_t> rows_of(const std::vector<uint64_t> &ps, size_t reps) {
    std::vector<uint64_t> r;
    for (size_t k = 0; k < reps; k++) r.insert(r.end(), ps.begin(), ps.end());
    return r;
}

static std::vector<uint64_t> first_primes(const Env &E, size_t L) {
    return std::vector<uint64_t>(E.primes.begin(), E.primes.begin() + L);
}

// a shared-a batch of n members at L limbs, b_i filled with tag + i and a with tag + 9
static void fill_batch(const Env &E, moai::SharedACiphertextBatch &b, size_t n, size_t L, uint64_t tag) {
    b.allocate(E.context, 1 + (E.nq - L), n, std::pow(2.0, 40), E.s);
    std::vector<uint64_t> v(L * E.N);
    for (size_t i = 0; i < n; i++) {
        fill(v, tag + i, E.N, first_primes(E, L));
        h2d(b.b_[i].get(), v);
    }
    fill(v, tag + 9, E.N, first_primes(E, L));
    h2d(b.a_.get(), v);
}

// a shared-a batch in the layout [n + 1][L][N] = (b_0 .. b_{n-1}, a)
static void dump_batch(const Env &E, const char *name, const moai::SharedACiphertextBatch &b) {
    const size_t L = b.size_Ql_, w = L * E.N;
    std::vector<uint64_t> all;
    all.reserve((b.n_ + 1) * w);
    for (size_t i = 0; i < b.n_; i++) {
        auto v = d2h(b.b_[i].get(), w);
        all.insert(all.end(), v.begin(), v.end());
    }
    auto a = d2h(b.a_.get(), w);
    all.insert(all.end(), a.begin(), a.end());
    emit(name, all, (b.n_ + 1) * L, E.N);
}

static PhantomCiphertext make_ct_env(const Env &E, uint64_t tag, size_t limbs) {
    PhantomCiphertext ct;
    ct.resize(E.context, 1 + (E.nq - limbs), 2, E.s);
    ct.set_scale(std::pow(2.0, 40));
    ct.set_ntt_form(true);
    std::vector<uint64_t> v(2 * limbs * E.N);
    fill(v, tag, E.N, rows_of(first_primes(E, limbs), 2));
    h2d(ct.data(), v);
    return ct;
}

static void load_key_env(const Env &E, const PhantomRelinKey &key, uint64_t tag) {
    std::vector<uint64_t *> ptrs(E.dnum);
    cudaDeviceSynchronize();
    cudaMemcpy(ptrs.data(), key.public_keys_ptr(), E.dnum * sizeof(uint64_t *), cudaMemcpyDeviceToHost);
    for (size_t d = 0; d < E.dnum; d++) {
        std::vector<uint64_t> v(2 * E.QP * E.N);
        fill(v, tag + d, E.N, rows_of(E.primes, 2));
        h2d(ptrs[d], v);
    }
}

// FmtSwitch forward and backward for groups of n at L limbs.  The format key rows live in the QlP
// basis (FmtSwitch.cuh:31-40): a_fmt[j] tag 400 + j, B_fmt[j][i] tag 500 + j n + i; backward key i
// digit d tag 600 + 10 i + d.  Inputs: ciphertext j tag 30 + j; the backward batch tags 50.. (fill_batch).
static void shared_fmt_records(const Env &E, size_t n, size_t L) {
    const size_t chain = 1 + (E.nq - L), QlP = L + E.np, pc = QlP * E.N;
    std::vector<uint64_t> qlp_rows = first_primes(E, L);
    qlp_rows.insert(qlp_rows.end(), E.primes.begin() + E.nq, E.primes.end());
    moai::SharedAFormatKey fk;
    fk.n_ = n;
    fk.chain_index_ = chain;
    fk.size_Ql_ = L;
    fk.size_P_ = E.np;
    fk.a_fmt_ = make_cuda_auto_ptr<uint64_t>(n * pc, E.s);
    fk.B_fmt_ = make_cuda_auto_ptr<uint64_t>(n * n * pc, E.s);
    std::vector<uint64_t> v(pc);
    for (size_t j = 0; j < n; j++) {
        fill(v, 400 + j, E.N, qlp_rows);
        h2d(fk.a_fmt_.get() + j * pc, v);
        for (size_t i = 0; i < n; i++) {
            fill(v, 500 + j * n + i, E.N, qlp_rows);
            h2d(fk.B_fmt_.get() + (j * n + i) * pc, v);
        }
    }
    for (size_t i = 0; i < n; i++) {
        fk.backward_keys_.emplace_back(E.sk.gen_relinkey(E.context));
        load_key_env(E, fk.backward_keys_[i], 600 + 10 * i);
    }
    std::vector<PhantomCiphertext> cts;
    for (size_t j = 0; j < n; j++) cts.push_back(make_ct_env(E, 30 + j, L));
    moai::SharedACiphertextBatch out;
    moai::fmt_switch_forward(E.context, cts, fk, out, E.s);
    char nm[64];
    snprintf(nm, sizeof nm, "fmt_fwd_n%zu_L%zu", n, L);
    dump_batch(E, nm, out);

    moai::SharedACiphertextBatch in;
    fill_batch(E, in, n, L, 50);
    std::vector<PhantomCiphertext> back;
    moai::fmt_switch_backward(E.context, in, fk, back, E.s);
    std::vector<uint64_t> all;
    for (auto &ct : back) {
        auto w = d2h(ct.data(), 2 * L * E.N);
        all.insert(all.end(), w.begin(), w.end());
    }
    snprintf(nm, sizeof nm, "fmt_bwd_n%zu_L%zu", n, L);
    emit(nm, all, n * 2 * L, E.N);
}

// Sh-Rot of a group of n at L limbs by `step` with a Sh-Galois key whose A_g has tag 700 + g and
// B_{g,i} tag 800 + g n + i (ShRotate.cuh:25-36); input batch tags 60.. (fill_batch)
static void shared_rot_record(const Env &E, size_t n, size_t L, int step) {
    moai::SharedAGaloisKey key;
    key.step_ = step;
    key.n_ = n;
    key.dnum_ = E.dnum;
    auto elts = get_elts_from_steps(std::vector<int>{step}, E.N);
    key.galois_elt_ = elts[0];
    key.tool_ = std::make_unique<PhantomGaloisTool>(elts, E.log_n, E.s, false);
    const size_t pc = E.QP * E.N;
    key.A_ = make_cuda_auto_ptr<uint64_t>(E.dnum * pc, E.s);
    key.B_ = make_cuda_auto_ptr<uint64_t>(E.dnum * n * pc, E.s);
    std::vector<uint64_t> v(pc);
    for (size_t g = 0; g < E.dnum; g++) {
        fill(v, 700 + g, E.N, E.primes);
        h2d(key.A_.get() + g * pc, v);
        for (size_t i = 0; i < n; i++) {
            fill(v, 800 + g * n + i, E.N, E.primes);
            h2d(key.B_.get() + (g * n + i) * pc, v);
        }
    }
    moai::SharedACiphertextBatch in, out;
    fill_batch(E, in, n, L, 60);
    moai::shared_a_rotate(E.context, in, key, out, E.s);
    char nm[64];
    snprintf(nm, sizeof nm, "shrot_n%zu_L%zu_s%d", n, L, step);
    printf(",\n  \"%s_elt\": %u", nm, (unsigned)elts[0]);
    dump_batch(E, nm, out);
}

static int run_shared(const Env &E, const std::string &which) {
    const bool tiny = which == "tiny";
    const size_t n = 4;
    // FmtSwitch at the bootstrap's input level (4 primes; 2 at N = 2^12), groups of 4 and 8
    const size_t L_fmt = tiny ? 2 : 4;
    shared_fmt_records(E, n, L_fmt);
    shared_fmt_records(E, 8, L_fmt);
    // Sh-Rot at the top level, one level below it (a short last digit) and at 3 primes
    shared_rot_record(E, n, E.nq, 1);
    shared_rot_record(E, n, E.nq - 1, 1);
    shared_rot_record(E, n, 3, -3);
    {   // shared_a_rescale_to_next_inplace at L = nq - 1 (tags 70..)
        moai::SharedACiphertextBatch b;
        fill_batch(E, b, n, E.nq - 1, 70);
        moai::shared_a_rescale_to_next_inplace(E.context, b, E.s);
        dump_batch(E, "shared_rescale", b);
    }
    {   // shared_a_modraise_inplace from one prime (tags 80..)
        moai::SharedACiphertextBatch b;
        fill_batch(E, b, n, 1, 80);
        moai::shared_a_modraise_inplace(E.context, b, E.s);
        dump_batch(E, "shared_modraise", b);
    }
    {   // shared_a_multiply_plain_inplace at 3 limbs (batch tags 90.., plaintext tag 98) and
        // shared_a_add_inplace of two batches (tags 110.. and 120..)
        const size_t L = 3;
        moai::SharedACiphertextBatch b;
        fill_batch(E, b, n, L, 90);
        PhantomPlaintext pt;
        pt.resize(L, E.N, E.s);
        pt.set_chain_index(1 + (E.nq - L));
        std::vector<uint64_t> v(L * E.N);
        fill(v, 98, E.N, first_primes(E, L));
        h2d(pt.data(), v);
        moai::shared_a_multiply_plain_inplace(E.context, b, pt, E.s);
        dump_batch(E, "shared_mulplain", b);
        moai::SharedACiphertextBatch x, y;
        fill_batch(E, x, n, L, 110);
        fill_batch(E, y, n, L, 120);
        moai::shared_a_add_inplace(E.context, x, y, E.s);
        dump_batch(E, "shared_add", x);
    }
    {   // complex slot-vector encode at the top level: slot j = unit(12, j) + i unit(13, j); the
        // record holds the NTT-form plaintext and the integer coefficients (the reference's own INTT
        // of limb 0, centred), all of them at N = 2^12, every 8th at N = 2^16
        const double scale = std::pow(2.0, tiny ? 40 : 46);
        std::vector<std::complex<double>> z(E.N / 2);
        for (size_t j = 0; j < z.size(); j++) z[j] = std::complex<double>(unit(12, j), unit(13, j));
        PhantomPlaintext pt;
        E.encoder.encode(E.context, z, scale, pt, 1, *global_variables::default_stream);
        auto v = d2h(pt.data(), E.nq * E.N);
        emit("encode_z", v, E.nq, E.N);
        auto c = make_cuda_auto_ptr<uint64_t>(E.N, E.s);
        cudaMemcpyAsync(c.get(), pt.data(), E.N * 8, cudaMemcpyDeviceToDevice, E.s);
        nwt_2d_radix8_backward_inplace(c.get(), E.context.gpu_rns_tables(), 1, 0, E.s);
        auto co = d2h(c.get(), E.N);
        const size_t stride = tiny ? 1 : 8;
        printf(",\n  \"encode_z_coeffs\": {\"scale_log2\": %d, \"stride\": %zu, \"values\": [", tiny ? 40 : 46, stride);
        for (size_t k = 0; k < E.N; k += stride) {
            int64_t x = co[k] > E.primes[0] / 2 ? -(int64_t)(E.primes[0] - co[k]) : (int64_t)co[k];
            printf("%s\"%lld\"", k ? ", " : "", (long long)x);
        }
        printf("]}");
    }
    printf("\n}\n");
    cudaDeviceSynchronize();
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// ---- timing of the reference's own calls (CUDA events on the evaluator's stream)

static double time_ms(cudaStream_t s, int warm, int reps, const std::function<void()> &fn) {
    for (int i = 0; i < warm; i++) fn();
    cudaDeviceSynchronize();
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
    for (int i = 0; i < reps; i++) fn();
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    cudaDeviceSynchronize();
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / reps;
}

// the per-ciphertext ct-pt loop of ct_pt_matrix_mul_wo_pre_single (Ct_pt_matrix_mul.cuh:188-303),
// call for call on the default stream: per output column, a scalar encode of each weight at the
// input's level and scale, multiply_plain into a new ciphertext, add_inplace into the accumulator,
// then rescale_to_next_inplace; one encoder and evaluator for the whole loop (the reference's
// single-thread region).  n_in inputs at L limbs, the first n_out output columns.
static double ctpt_loop_ms(const Env &E, size_t n_in, size_t n_out, size_t L) {
    std::vector<PhantomCiphertext> X;
    X.reserve(n_in);
    const size_t words = 2 * L * E.N;
    for (size_t j = 0; j < n_in; j++) {
        if (j < 4) {
            X.push_back(make_ct_env(E, 20 + j, L));
        } else {  // distinct buffers, contents copied on the device
            PhantomCiphertext ct;
            ct.resize(E.context, X[0].chain_index(), 2, E.s);
            ct.set_scale(X[0].scale());
            ct.set_ntt_form(true);
            cudaMemcpyAsync(ct.data(), X[j % 4].data(), words * 8, cudaMemcpyDeviceToDevice, E.s);
            X.push_back(std::move(ct));
        }
    }
    cudaDeviceSynchronize();
    PhantomCKKSEncoder penc(E.context);
    moai::Encoder enc(&E.context, &penc);
    moai::Evaluator ev(&E.context, &penc);
    std::vector<PhantomCiphertext> out;
    auto run = [&](size_t cols) {
        out.clear();
        for (size_t i = 0; i < cols; i++) {
            PhantomPlaintext p0;
            enc.encode(weight(8, i), X[0].chain_index(), X[0].scale(), p0);
            PhantomCiphertext acc;
            ev.multiply_plain(X[0], p0, acc);
            for (size_t j = 1; j < n_in; j++) {
                PhantomPlaintext pj;
                enc.encode(weight(8, j * 768 + i), X[j].chain_index(), X[j].scale(), pj);
                PhantomCiphertext tmp;
                ev.multiply_plain(X[j], pj, tmp);
                ev.add_inplace(acc, tmp);
            }
            ev.rescale_to_next_inplace(acc);
            out.push_back(std::move(acc));
        }
    };
    run(1);  // warm-up: one column
    cudaDeviceSynchronize();
    auto t0 = std::chrono::steady_clock::now();
    run(n_out);
    cudaDeviceSynchronize();
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

static int run_time(const Env &E, const std::string &which, int ctpt_cols) {
    PhantomCiphertext A = make_ct_env(E, 1, E.nq), B = make_ct_env(E, 2, E.nq);
    const int warm = 3, reps = 20;
    const cudaStream_t s = E.s;
    double ntt = time_ms(s, warm, reps, [&] {
        E.ev.transform_from_ntt_inplace(A);
        E.ev.transform_to_ntt_inplace(A);
    });
    double rot = time_ms(s, warm, reps, [&] { E.ev.rotate_vector_inplace(A, 1, E.gk); });
    double mrr = time_ms(s, warm, reps, [&] {
        PhantomCiphertext t;
        E.ev.multiply(A, B, t);
        E.ev.relinearize_inplace(t, E.rk);
        E.ev.rescale_to_next_inplace(t);
    });
    printf(",\n  \"time\": {\"limbs\": %zu, \"warmup\": %d, \"reps\": %d, \"ntt_inv_fwd_ms\": %.4f, "
           "\"rotate1_ms\": %.4f, \"mul_relin_rescale_ms\": %.4f, \"chain_ms\": %.4f",
           E.nq, warm, reps, ntt, rot, mrr, ntt + rot + mrr);
    if (ctpt_cols > 0) {
        const size_t n_in = 768, L = 13;
        double ms = ctpt_loop_ms(E, n_in, (size_t)ctpt_cols, L);
        printf(", \"ctpt_loop\": {\"n_in\": %zu, \"n_out\": %d, \"limbs\": %zu, \"threads\": 1, \"ms\": %.3f}",
               n_in, ctpt_cols, L, ms);
    }
    printf("}\n}\n");
    cudaDeviceSynchronize();
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int main(int argc, char **argv) {
    setvbuf(stdout, nullptr, _IONBF, 0);  // a failure late in a run keeps the records printed before it
    std::string which = argc > 1 ? argv[1] : "tiny";
    std::string mode = argc > 2 ? argv[2] : "golden";
    const int ctpt_cols = argc > 3 ? atoi(argv[3]) : 0;
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

    const std::string set_name = mode == "shared" ? "shared_" + which : which;
    printf("{\n  \"params\": {\"name\": \"%s\", \"log_n\": %d, \"nq\": %zu, \"np\": %zu, \"dnum\": %zu, \"primes\": [",
           set_name.c_str(), log_n, nq, np, dnum);
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

    if (mode == "shared" || mode == "time") {
        Env E{context, encoder, enc, ev, sk, rk, gk, primes, N, nq, np, dnum, QP, log_n, s};
        try {
            return mode == "shared" ? run_shared(E, which) : run_time(E, which, ctpt_cols);
        } catch (const std::exception &e) {
            fprintf(stderr, "ref_golden %s %s: %s\n", which.c_str(), mode.c_str(), e.what());
            return 2;
        }
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
