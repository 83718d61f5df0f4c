// C++ host API of the B200 CKKS core: the evaluator, key material and S2C-first
// (shared-a) batched bootstrapping that the MOAI driver calls, over the C ABI of
// include/shmoai_ckks.h.
//
// Mirrors the reference's host classes (src/include/source/ckks_evaluator_parallel.cuh:13-680:
// moai::Encoder / Encryptor / Evaluator / Decryptor / CKKSEvaluator) and
// BatchBootstrapper::{prepare, prepare_shared_keys, bootstrap_ordinary_s2c_first,
// bootstrap_shared_a_s2c_first} (src/include/source/bootstrapping/BatchBootstrap.cuh:470-820),
// with two differences that the B200 design asks for:
//   * a Ciphertext is a BATCH [count][size][L][N] (one launch per operation for the
//     whole batch); a shared-a batch is the same type with `shared` set, holding
//     [groups][members + 1][L][N] = (b_0 .. b_{n-1}, a) per group
//     (SharedACiphertextBatch, SharedACiphertext.cuh:22-99);
//   * scales are tracked exactly (products and quotients of primes and encoded
//     constants), and adding ciphertexts whose scales differ throws, instead of the
//     reference's assumed-nominal scales and *_reduced_error level alignment.
// Errors throw shmoai::Error with the C ABI's message.
#pragma once

#include <complex>
#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../shmoai_ckks.h"

namespace shmoai {

using cplx = std::complex<double>;

struct Error : std::runtime_error {
    explicit Error(const std::string &msg, int code_ = SHM_EINVAL) : std::runtime_error(msg), code(code_) {}
    int code;  // the SHM_E* status behind it
};

class Context;

// Move-only owner of shm_malloc'd device words.
class DeviceBuffer {
   public:
    DeviceBuffer() = default;
    DeviceBuffer(const Context &c, size_t words);
    ~DeviceBuffer();
    DeviceBuffer(DeviceBuffer &&o) noexcept;
    DeviceBuffer &operator=(DeviceBuffer &&o) noexcept;
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    uint64_t *data() const { return p_; }
    size_t words() const { return words_; }
    DeviceBuffer clone() const;
    // free through `c` (a view of the same context) from now on; the caller has made
    // sure no work on the allocating stream still uses the buffer
    void rebind(const Context &c) { ctx_ = &c; }

   private:
    const Context *ctx_ = nullptr;
    uint64_t *p_ = nullptr;
    size_t words_ = 0;
};

// Ring parameters, prime chain Q (nq primes) + special primes P (np), device, stream.
class Context {
   public:
    Context(uint32_t log_n, const std::vector<int> &bits, uint32_t n_special, int device = 0, void *stream = nullptr);
    Context(uint32_t log_n, const std::vector<uint64_t> &primes, uint32_t n_special, int device = 0,
            void *stream = nullptr);
    // a non-owning view of `base` (same device tables) whose operations run on `stream`;
    // `base` must outlive it, and it must outlive every buffer allocated through it
    Context(const Context &base, void *stream);
    ~Context();
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;

    shm_context *handle() const { return h_; }
    void *stream() const { return stream_; }
    void check(int rc) const;  // throws Error unless rc == SHM_OK
    void synchronize() const;
    size_t slot_count() const { return n / 2; }
    // reference chain index of a ciphertext with L primes (context.cu:148-174)
    size_t chain_index(uint32_t L) const { return nq - L + 1; }

    uint32_t log_n = 0, n = 0, nq = 0, np = 0, dnum = 0;
    std::vector<uint64_t> primes;

   private:
    void init();
    shm_context *h_ = nullptr;
    void *stream_ = nullptr;
    bool owner_ = true;
};

struct Plaintext {
    DeviceBuffer data;  // [L][N], NTT form
    uint32_t L = 0;
    double scale = 1.0;
    size_t coeff_modulus_size() const { return L; }
};

// A batch of ciphertexts [count][size][L][N] (NTT form), or, with `shared`, a batch
// of shared-a groups [count][size][L][N] with size = members + 1.
struct Ciphertext {
    DeviceBuffer data;
    uint32_t count = 0, size = 2, L = 0;
    double scale_ = 1.0;
    bool shared = false;

    double scale() const { return scale_; }
    void set_scale(double s) { scale_ = s; }
    size_t coeff_modulus_size() const { return L; }
    uint32_t members() const { return shared ? size - 1 : 1; }
    size_t polys() const { return (size_t)count * size; }
};

class Encoder {
   public:
    explicit Encoder(const Context &c);
    size_t slot_count() const { return c_.n / 2; }
    // unrounded coefficients of the polynomial whose slots are z * scale (z padded with 0), by
    // the host's FFT: the restatement the device encoder (shm_encode) is checked against
    std::vector<double> encode_float(const cplx *z, size_t len, double scale) const;
    // rounded (half to even) integer coefficients; |c| < 2^62 or Error (shm_encode, FP64 on
    // the device)
    std::vector<int64_t> encode_coeffs(const cplx *z, size_t len, double scale) const;
    // the same for several slot vectors at once, into device memory [rows][N] (int64 words)
    void encode_rows(const std::vector<std::vector<cplx>> &z, double scale, uint64_t *coeffs) const;
    // device integer coefficients [n_polys][N] -> NTT-form residues [n_polys][L][N], or over QlP
    void lift(const uint64_t *coeffs, size_t n_polys, uint32_t L, uint64_t *out) const;
    void lift_ext(const uint64_t *coeffs, size_t n_polys, uint32_t L, uint64_t *out) const;
    Plaintext encode(const std::vector<cplx> &z, uint32_t L, double scale) const;
    // the same plaintext over the extended basis QlP: L + n_p limbs (the Q limbs, then the
    // special primes); its first L limbs are encode(z, L, scale).  L stays the Q limb count.
    Plaintext encode_ext(const std::vector<cplx> &z, uint32_t L, double scale) const;
    // a constant: the single coefficient round(value * scale)
    // (moai::Encoder::encode(double), ckks_evaluator_parallel.cuh:73-92)
    Plaintext encode(double value, uint32_t L, double scale) const;
    std::vector<cplx> decode(const std::vector<double> &coeffs, double scale) const;
    // several coefficient vectors (real, centred) at once on the device (shm_decode)
    std::vector<std::vector<cplx>> decode_rows(const std::vector<std::vector<double>> &coeffs, double scale) const;
    // signed integer coefficients [n_polys][N] (host) -> NTT-form residues [n_polys][L][N] at `out`
    void upload(const int64_t *coeffs, size_t n_polys, uint32_t L, uint64_t *out) const;
    // ... to [n_polys][L + n_p][N] over the extended basis QlP
    void upload_ext(const int64_t *coeffs, size_t n_polys, uint32_t L, uint64_t *out) const;

   private:
    void fft(std::vector<cplx> &a, bool inverse) const;
    const Context &c_;
    std::vector<uint32_t> exps_;  // 5^j mod 2N
    std::vector<cplx> roots_;     // exp(2 pi i k / 2N)
};

// The keys of one group size of shared-a batches.
struct SharedAKeys {
    uint32_t members = 0;
    std::map<uint32_t, DeviceBuffer> galois;  // element -> [dnum][members + 1][QP][N]
    DeviceBuffer format;                      // [members][members + 1][QP][N]
    std::vector<DeviceBuffer> backward;       // members x [dnum][2][QP][N] (s'_i -> s)
};

// Secret key, auxiliary secrets and every evaluation key (the reference's
// PhantomSecretKey key generation, secretkey.cu:328-646, and SharedAKeyGen,
// FmtSwitch.cuh:235-305 / ShRotate.cu:54-162 / FmtSwitch.cu:165-270), plus symmetric
// encryption and decryption.  Deterministic in `seed`.
class KeyGenerator {
   public:
    KeyGenerator(const Context &c, uint32_t hamming_weight = 192, uint64_t seed = 0x5EED);
    const DeviceBuffer &secret() const { return s_; }  // [QP][N] NTT form
    DeviceBuffer switching_key(const DeviceBuffer &s_new);  // [dnum][2][QP][N]: s_new -> s
    DeviceBuffer relin_key();
    // [2][QP][N] = (e - a s, a) in NTT form (gen_publickey, secretkey.cu:524-537)
    DeviceBuffer public_key();
    DeviceBuffer galois_key(uint32_t elt);
    std::map<uint32_t, DeviceBuffer> galois_keys(const std::vector<uint32_t> &elts);

    void gen_aux_secrets(uint32_t members, uint32_t hamming_weight = 192);
    DeviceBuffer shared_galois_key(uint32_t elt);
    DeviceBuffer format_key();
    std::vector<DeviceBuffer> backward_keys();
    SharedAKeys shared_keys(uint32_t members, const std::vector<uint32_t> &elts, uint32_t hamming_weight = 192);

    // z: count rows of up to N/2 slot values
    Ciphertext encrypt(const std::vector<std::vector<cplx>> &z, double scale, uint32_t L);
    // centred limb-0 coefficients of every member (exact while |m| < q0 / 2)
    std::vector<std::vector<double>> decrypt_coeffs(const Ciphertext &ct);
    std::vector<std::vector<cplx>> decrypt(const Ciphertext &ct);

    // signed coefficients of the secret and of the auxiliary secrets of shared-a groups
    const std::vector<int64_t> &secret_coeffs() const { return s_coeffs_; }
    const std::vector<std::vector<int64_t>> &aux_secret_coeffs() const { return aux_coeffs_; }
    // replace the secret and the auxiliary secrets (keys made earlier are not touched), e.g.
    // with ones read from a key stream or the reference's secret-key text
    void import_secrets(const std::vector<int64_t> &s, const std::vector<std::vector<int64_t>> &aux);

   private:
    uint64_t next_seed();
    std::vector<int64_t> ternary(uint32_t hamming_weight);
    DeviceBuffer ntt_qp(const std::vector<int64_t> &coeffs) const;  // [QP][N]
    DeviceBuffer automorph_ntt(const DeviceBuffer &s_ntt, uint32_t elt) const;  // s(X^elt), [QP][N] NTT form
    // B_{d,row} += unit * s (unit: residues over QP)
    struct KeyTerm {
        uint32_t row;
        std::vector<uint64_t> unit;
        const DeviceBuffer *s;
    };
    // [D][olds + 1][QP][N]: digit d = (B_{d,0} .. B_{d,n-1}, A_d), B_{d,i} = e - A_d olds[i] + terms
    DeviceBuffer multi_key(const std::vector<const DeviceBuffer *> &olds, const std::vector<std::vector<KeyTerm>> &adds);
    std::vector<uint64_t> p_units(int digit) const;

    const Context &c_;
    Encoder enc_;
    uint64_t seed_, ctr_ = 0;
    std::vector<int64_t> s_coeffs_;
    DeviceBuffer s_;
    std::vector<std::vector<int64_t>> aux_coeffs_;
    std::vector<DeviceBuffer> aux_;
};

// Public-key encryption (PhantomPublicKey::encrypt_asymmetric and
// encrypt_zero_asymmetric_internal, thirdparty/phantom-fhe/src/secretkey.cu:15-217): with
// pk = (e - a s, a) over QP, a ternary u and CBD errors e0, e1 over QP, the ciphertext is the
// ModDown to Q of u pk + (e0, e1), limbs dropped to L, plus the encoded message on c0.  The
// reference runs the ModDown only from the key level to the top data level (chain index 1) and
// encrypts only there in practice; below the top level this class drops limbs after it.
// Deterministic in `seed` (counter-based samplers, like KeyGenerator).
class PublicEncryptor {
   public:
    PublicEncryptor(const Context &c, DeviceBuffer pk, uint64_t seed = 0xE0C0);
    Ciphertext encrypt(const std::vector<std::vector<cplx>> &z, double scale, uint32_t L);
    // an encoded plaintext (moai::Encryptor::encrypt(plain, ct)): one ciphertext at pt.L, pt.scale
    Ciphertext encrypt(const Plaintext &pt);
    // count encryptions of zero at L primes
    Ciphertext encrypt_zero(uint32_t count, uint32_t L, double scale);
    const DeviceBuffer &public_key() const { return pk_; }

   private:
    const Context &c_;
    Encoder enc_;
    DeviceBuffer pk_;  // [2][QP][N] NTT form
    uint64_t seed_, ctr_ = 0;
};

// ---- the MOAI packing of a batch of inputs (src/include/source/matrix_mul/Batch_encode_encrypt.cuh)

// Column-interleaved packing (batch_input, Batch_encode_encrypt.cuh:12-43): X holds num_X
// matrices of num_row x num_col values, X[(j * num_row + k) * num_col + i] = input j, row k,
// column i; column i becomes one ciphertext whose slot num_X * k + j holds X_j[k][i] (num_X *
// num_row <= N / 2, the other slots 0).  All columns are encoded in one batch on the device and
// encrypted with the public key at L primes; the result is a batch of num_col ciphertexts.
Ciphertext batch_input(PublicEncryptor &enc, const std::vector<double> &X, uint32_t num_X, uint32_t num_row,
                       uint32_t num_col, double scale, uint32_t L);
// The matching slot mask (bias_vec, Batch_encode_encrypt.cuh:45-56): slot j * num_X + i is 1 for
// the first lengths[i] rows of input i, 0 elsewhere.
std::vector<int> bias_vec(const std::vector<int> &lengths, uint32_t num_X, uint32_t num_row);

// moai::Encryptor / moai::Decryptor names over the key generator's secret.
class Encryptor {
   public:
    explicit Encryptor(KeyGenerator &kg) : kg_(kg) {}
    Ciphertext encrypt(const std::vector<std::vector<cplx>> &z, double scale, uint32_t L) {
        return kg_.encrypt(z, scale, L);
    }

   private:
    KeyGenerator &kg_;
};

class Decryptor {
   public:
    explicit Decryptor(KeyGenerator &kg) : kg_(kg) {}
    std::vector<std::vector<cplx>> decrypt(const Ciphertext &ct) { return kg_.decrypt(ct); }

   private:
    KeyGenerator &kg_;
};

// moai::Evaluator over batches, with exact scale tracking.
class Evaluator {
   public:
    Evaluator(const Context &c, const Encoder &enc);
    const Context &context() const { return c_; }
    const Encoder &encoder() const { return enc_; }

    // keys (not owned)
    const DeviceBuffer *relin_key = nullptr;
    const std::map<uint32_t, DeviceBuffer> *galois_keys = nullptr;
    const SharedAKeys *shared_keys = nullptr;

    static bool same_scale(double a, double b, double rel = 1e-11);

    Ciphertext mod_switch_to(const Ciphertext &a, uint32_t L) const;  // drop limbs
    Ciphertext add(const Ciphertext &a, const Ciphertext &b) const;
    Ciphertext sub(const Ciphertext &a, const Ciphertext &b) const;
    Ciphertext negate(const Ciphertext &a) const;
    Ciphertext multiply_plain(const Ciphertext &a, const Plaintext &p) const;
    Ciphertext multiply_int(const Ciphertext &a, int64_t k) const;
    Ciphertext add_const(const Ciphertext &a, double c) const;
    Ciphertext rescale_to_next(const Ciphertext &a) const;
    // a * round(c * T) with T = target * q / a.scale, then rescale: result at exactly `target`
    Ciphertext multiply_const(const Ciphertext &a, double c, double target) const;
    Ciphertext multiply_const(const Ciphertext &a, double c) const { return multiply_const(a, c, a.scale_); }
    // a * round(c * T) without rescale; the result's scale is a.scale * T
    Ciphertext multiply_const_unscaled(const Ciphertext &a, double c, double T) const;
    Ciphertext adjust(const Ciphertext &a, uint32_t L, double scale) const;
    Ciphertext multiply(const Ciphertext &a, const Ciphertext &b, bool rescale = true) const;
    // the tensor product only: a size-3 batch at scale a.scale * b.scale (the reference's
    // multiply before relinearize_inplace, evaluate.cu:350-402); it may be rescaled, added
    // to (also to size-2 batches) and relinearised later
    Ciphertext multiply_lazy(const Ciphertext &a, const Ciphertext &b) const;
    Ciphertext relinearize(const Ciphertext &a) const;  // size 3 -> 2 (evaluate.cu:1358-1390)
    // size 3 at L -> size 2 at L - 1 with one ModDown by q_{L-1} P (shm_relinearize_rescale):
    // relinearize then rescale_to_next up to a few units per coefficient, one forward NTT fewer
    Ciphertext relinearize_rescale(const Ciphertext &a) const;
    // sum_i w_i X_i + w0 (added to c0) at L primes in one pass, the X_i read at their first L
    // limbs; w_i and w0 are integers held exactly by doubles; the result is given `scale`
    // (the terms' common scale times the weights' factor)
    Ciphertext linear_combination(const std::vector<const Ciphertext *> &X, const std::vector<double> &w, double w0,
                                  uint32_t L, double scale) const;
    Ciphertext square(const Ciphertext &a) const { return multiply(a, a); }
    // sum_k X_k * P_k (same level and scale), one launch; result scale X.scale * P.scale
    Ciphertext multiply_plain_accumulate(const std::vector<const Ciphertext *> &X,
                                         const std::vector<const Plaintext *> &P) const;

    uint32_t galois_elt(int step) const;
    Ciphertext rotate_vector(const Ciphertext &a, int step) const;
    std::map<int, Ciphertext> rotate_many(const Ciphertext &a, const std::vector<int> &steps) const;
    Ciphertext complex_conjugate(const Ciphertext &a) const;
    // times i (sign +1) or -i, through the monomial X^(N/2): exact, no level
    Ciphertext multiply_i(const Ciphertext &a, int sign = 1) const;
    Ciphertext mod_raise(const Ciphertext &a1, uint32_t L) const;  // 1 prime -> L primes, centred lift
    Ciphertext concat(const Ciphertext &a, const Ciphertext &b) const;
    Ciphertext slice(const Ciphertext &a, uint32_t first, uint32_t count) const;

    Ciphertext to_shared(const Ciphertext &a, uint32_t members) const;  // FmtSwitch forward
    Ciphertext from_shared(const Ciphertext &a) const;                  // FmtSwitch backward

    // Rotation-free ct-pt matmul Y[o] = sum_i X[i] * W[i][o] (W: [n_in][n_out] integers, the
    // encoded weights round(w * w_scale)) followed by a rescale: the reference's
    // multiply_plain + add_inplace + rescale loop (Ct_pt_matrix_mul.cuh:112-158).  Tensor
    // cores (exact residue GEMMs) or the CUDA-core kernel; both exact.
    Ciphertext ctpt_matmul(const Ciphertext &X, const std::vector<int64_t> &W, uint32_t n_out, double w_scale,
                           bool tensor_cores = true) const;
    // The masked projection (ct_pt_matrix_mul_wo_pre_w_mask, Ct_pt_matrix_mul.cuh:846-986):
    // Y[o] = mask * sum_i X[i] W[i][o] slot-wise.  The reference encodes W[i][o] * mask as its own
    // slot-vector plaintext for every (i, o) (n_in * n_out encodes, one level); here the weights
    // stay scalars (ctpt_matmul, one level) and the mask is encoded once, at the product's level
    // with the next prime as its scale, and multiplies every output before a second rescale
    // (two levels, output scale X.scale * w_scale / q exactly as ctpt_matmul's).  mask: N/2 slots.
    Ciphertext ctpt_matmul_masked(const Ciphertext &X, const std::vector<int64_t> &W, uint32_t n_out,
                                  double w_scale, const std::vector<double> &mask, bool tensor_cores = true) const;

    // out[c] = sum_t A[t][c] x B[t][c] as size-3 ciphertexts, the products summed before one
    // reduction (shm_multiply_accumulate); every B[t] of one member is broadcast over the batch.
    // Equal to multiply_lazy of every pair followed by add.  Terms at different levels are
    // brought to the lowest.
    Ciphertext multiply_accumulate(const std::vector<const Ciphertext *> &A,
                                   const std::vector<const Ciphertext *> &B) const;
    // sum over the members j of X_j x W_j: one size-3 ciphertext
    Ciphertext sum_of_products(const Ciphertext &X, const Ciphertext &W) const;

    // frees the scratch buffer that key switches, rescales and matmuls share (it grows to the
    // largest request and is kept); the next such call allocates it again
    void release_workspace() const;

   private:
    std::vector<uint64_t> residues(double integral, uint32_t L) const;
    std::vector<Ciphertext> automorphisms(const Ciphertext &a, const std::vector<uint32_t> &elts) const;
    uint64_t *ws(size_t bytes) const;
    Ciphertext like(const Ciphertext &a, uint32_t L) const;
    const Plaintext &monomial_half() const;

    const Context &c_;
    const Encoder &enc_;
    mutable DeviceBuffer ws_;
    mutable Plaintext mono_;
};

// ---- polynomial operators on ciphertext batches (chebyshev.cpp): the BERT layer's
// non-linear functions as Chebyshev series (src/include/source/non_linear_func/)

// coefficients c_0 .. c_deg of the interpolant of f at the deg + 1 Chebyshev nodes of [lo, hi]
std::vector<double> chebyshev_interpolant(const std::function<double(double)> &f, double lo, double hi, int deg);
// sum_k c_k T_k(u), u = (2 x - hi - lo) / (hi - lo), at x's scale; one level for u, then the
// basis and the baby-step giant-step tree (degree 24: 6 levels in all); approximates only on
// [lo, hi]
Ciphertext evaluate_chebyshev(const Evaluator &ev, const Ciphertext &x, const std::vector<double> &c, double lo,
                              double hi);
double gelu_exact(double x);  // x Phi(x) = x (1 + erf(x / sqrt 2)) / 2
// gelu_cheb's degree-24 near-minimax series on [-19.5, 12.5] (gelu_other.cuh:258-300), and
// GELU by it: 6 levels (gelu_cheb takes 7); inputs outside the interval are not approximated.  The scales stay
// near the primes when the levels it uses have primes of about the input scale's size
// (the chain's 46-bit primes at scale 2^46).
const std::vector<double> &gelu_series();
Ciphertext gelu(const Evaluator &ev, const Ciphertext &x);

struct BootstrapParams {
    double scale = 70368744177664.0;  // 2^46
    uint32_t input_level = 4;         // primes of the input (S2C-first)
    int K = 25;                       // EvalMod range
    int degree = 47;                  // Chebyshev degree
    int double_angles = 3;
    double F = 1.0 / 16;  // amplitude factor of SlotToCoeff (Bootstrapper.cuh:31)
    // baby-step count g1 of each slot-transform layer (S2C 0-2, C2S 3-5); 0 = the power of two
    // nearest above sqrt(diagonals); BatchBootstrapper::tune sets them
    int bsgs_g1[6] = {0, 0, 0, 0, 0, 0};
};

class LinearTransform;

// ------------------------------------------------------------------ CUDA graphs

// One recorded batch of device work, replayed with a single launch.  Graph(base, fn) makes a
// private stream, a view of base's context on it and an evaluator over the view with base's
// keys, runs fn(ev) once as is (workspaces grow, lazily built tables fill), then once under
// stream capture.  launch() replays the capture on base's stream.  fn must read and write
// only buffers that outlive the graph, free everything it allocates, and allocate the same
// sizes on every run.  No reference counterpart: the reference launches every kernel from
// the host per call.
class Graph {
   public:
    Graph(const Evaluator &base, const std::function<void(const Evaluator &ev)> &fn);
    ~Graph();
    Graph(const Graph &) = delete;
    Graph &operator=(const Graph &) = delete;
    void launch() const;
    uint64_t kernels() const;

   private:
    const Context &base_;
    void *stream_ = nullptr;
    std::unique_ptr<Context> view_;
    std::unique_ptr<Encoder> enc_;
    std::unique_ptr<Evaluator> ev_;
    shm_graph *g_ = nullptr;
};

// One autotuning decision: the candidates, their milliseconds (measured for the kernel
// tiles, modelled from measured rotation costs for the BSGS splits) and the pick.
// the softmax's building blocks (softmax.cuh:23-118): exp(x) by (1 + x/128)^128 (8 levels) and
// 1/x for x in (0, 2) by prod_{i <= iter} (1 + (1 - x)^(2^i)) (iter + 1 levels)
Ciphertext exp_approx(const Evaluator &ev, const Ciphertext &x);
Ciphertext inverse_approx(const Evaluator &ev, const Ciphertext &x, int iter);
// 1/sqrt(x) for LayerNorm (invert_sqrt, layernorm.cuh:708-897): a linear first guess,
// d_newt Newton steps and d_gold Goldschmidt steps (the reference uses 4 and 2)
Ciphertext inv_sqrt_approx(const Evaluator &ev, const Ciphertext &x, int d_newt = 4, int d_gold = 2);
// the sum of a batch's ciphertexts (one ciphertext), and one batch made of several
Ciphertext batch_sum(const Evaluator &ev, const Ciphertext &x);
Ciphertext batch_gather(const Evaluator &ev, const std::vector<Ciphertext> &parts);
// the same, releasing each part once it is copied (parts is left empty)
Ciphertext batch_gather(const Evaluator &ev, std::vector<Ciphertext> &&parts);
Ciphertext batch_broadcast(const Evaluator &ev, const Ciphertext &one, uint32_t count);  // count copies
// LayerNorm over the hidden columns of the column packing, one column per ciphertext of the
// batch (layernorm, layernorm.cuh:899-): gamma_i (x_i - mean) / sqrt(var) + beta_i with the
// inverse square root above; 2 (d_newt + d_gold) + 8 levels
// var_scale c > 0 brings the variance into the inverse square root's first-guess range: the
// iteration runs on c var (the factor joins the 1/d of the mean of squares) and sqrt(c) joins
// gamma, so no level is added (the reference's guess line suits variances of about 10..1000)
Ciphertext layernorm(const Evaluator &ev, const Ciphertext &x, const std::vector<double> &gamma,
                     const std::vector<double> &beta, int d_newt = 4, int d_gold = 2, double var_scale = 1.0);
// the same, releasing x once its centred columns are formed (x is left empty)
Ciphertext layernorm(const Evaluator &ev, Ciphertext &&x, const std::vector<double> &gamma,
                     const std::vector<double> &beta, int d_newt = 4, int d_gold = 2, double var_scale = 1.0);
// attention's ciphertext-ciphertext product in the column packing (ct_ct_matrix_mul_colpacking,
// Ct_ct_matrix_mul.cuh:10-120): X and W batches of the same count; output batch of `rows`,
// out_i = sum_j X_j * rot(W_j, i * num_batch) relinearised and rescaled (1 level); needs the
// Galois keys of the steps i * num_batch
// (with keys: the Galois keys are made from that generator a chunk of steps at a time and
// released, instead of read from ev.galois_keys)
Ciphertext ct_ct_matmul_colpacking(const Evaluator &ev, const Ciphertext &X, const Ciphertext &W, uint32_t rows,
                                   uint32_t num_batch, KeyGenerator *keys = nullptr);

// attention's ct-ct product in the diagonal packing (ct_ct_matrix_mul_diagpacking,
// Ct_ct_matrix_mul.cuh:182-): X holds the col_X = X.count diagonals, W the col_W = W.count
// columns; baby-step giant-step with g = ceil(sqrt(col_X)), b = ceil(col_X / g): X's members
// rotated by (col_X - i g) num_batch per giant step i, W's by j num_batch per baby step j,
// products summed and relinearised-rescaled per giant step, giant-step results rotated by
// j g num_batch and added (1 level); needs the Galois keys of those steps
Ciphertext ct_ct_matmul_diagpacking(const Evaluator &ev, const Ciphertext &X, const Ciphertext &W,
                                    uint32_t num_batch);

// the attention block's softmax with its masks (softmax, softmax.cuh:119-): the batch's members
// are the diagonals, bias_vec (one 0/1 per slot) marks the valid token slots, input_num the
// reference's band; shifts by -8.1, exp, mask subtraction, the inverse of the sum (iter
// steps) times each member; iter + 10 levels
Ciphertext softmax_attention(const Evaluator &ev, const Ciphertext &x, const std::vector<int> &bias_vec,
                             int input_num, int iter);
// the same softmax in two parts around a bootstrap of the members' sum (softmax_boot,
// softmax.cuh:512-): the shifted, exponentiated and masked members (8 levels), then, given the
// sum (refreshed by the caller), its inverse times every member (iter + 2 levels of the sum)
Ciphertext softmax_attention_numerators(const Evaluator &ev, const Ciphertext &x, const std::vector<int> &bias_vec,
                                        int input_num);
Ciphertext softmax_attention_finish(const Evaluator &ev, const Ciphertext &e, const Ciphertext &sum, int iter);
// softmax over the members of a batch (softmax.cuh:119-, without the attention layout's masks):
// e_i / sum_j e_j with e_i = exp_approx(x_i - shift) and the sum's inverse by inverse_approx on
// sum_scale * sum_j e_j, which the caller brings into (0, 2); iter + 12 levels
Ciphertext softmax_batch(const Evaluator &ev, const Ciphertext &x, double shift, double sum_scale, int iter);

// A CUDA graph of evaluate_chebyshev(ev, in, c, lo, hi) and the output batch every launch
// rewrites (write the next input into `in` between launches; `in` must outlive the graph).
std::unique_ptr<Graph> capture_chebyshev(const Evaluator &ev, const Ciphertext &in, const std::vector<double> &c,
                                         double lo, double hi, Ciphertext &out);

struct TuneRecord {
    std::string knob;
    std::vector<std::string> candidates;
    std::vector<double> ms;
    size_t chosen = 0;
};

// S2C-first batched bootstrapping, ordinary and shared-a (BatchBootstrap.cuh:674-819).
class BatchBootstrapper {
   public:
    BatchBootstrapper(Evaluator &ev, BootstrapParams p = BootstrapParams());
    ~BatchBootstrapper();
    // encode the slot-transform diagonals (resident) and the EvalMod polynomial
    void prepare();
    std::vector<int> rotation_steps() const;
    std::vector<uint32_t> galois_elts() const;
    // the shared-a keys of groups of `members` for this bootstrapper's rotations
    SharedAKeys prepare_shared_keys(KeyGenerator &kg, uint32_t members, uint32_t hamming_weight = 192) const;
    // The prepared diagonals are read-only, so any evaluator over the same context (for
    // instance one per serving slot, each on its own stream) may run the pipeline;
    // `ev` defaults to the one the bootstrapper was built with.
    Ciphertext bootstrap_ordinary_s2c_first(const Ciphertext &ct, const Evaluator *ev = nullptr) const;
    // groups of `members` consecutive ciphertexts; needs ev.shared_keys for that size
    Ciphertext bootstrap_shared_a_s2c_first(const Ciphertext &ct, uint32_t members,
                                            const Evaluator *ev = nullptr) const;
    // The original per-ciphertext C2S-first form (Bootstrapper::bootstrap_3 / bootstrap_full_3,
    // Bootstrapper.cu:3606-3627, 3889-3903): input at one prime (or brought there; scale Delta),
    // ModRaise to the top, CoeffToSlot, EvalMod, then SlotToCoeff at EvalMod's output level (its
    // diagonals are encoded there on the first call; make that call before any graph capture).
    // Ordinary ciphertexts, any batch size; the output has the input's slots at scale Delta.
    Ciphertext bootstrap_c2s_first(const Ciphertext &ct, const Evaluator *ev = nullptr) const;
    // EvalMod of ciphertexts holding t / K: c_fin * sin(2 pi t) read at scale Delta
    Ciphertext evalmod(const Ciphertext &x, const Evaluator *ev = nullptr) const;
    // Autotuning for batches of `count` ciphertexts (members per shared-a group, 0 =
    // ordinary): the NTT tile and, for shared-a, the Sh-Rot inner-product chunk (timed on
    // scratch data), the NTT tile again by a hoisted rotation of the batch at the top level
    // under each tile (record "ntt_tile (hoisted rotation, top level)", the tile kept; only
    // where the knobs time real kernels), then each slot-transform layer's BSGS split,
    // modelled from a hoisted ModUp and a per-step key switch timed at the layer's level;
    // re-prepares the layers.
    // The split decides the rotation steps, so call it before generating Galois keys.
    std::vector<TuneRecord> tune(uint32_t count, uint32_t members);
    // a stored split (BootstrapParams::bsgs_g1 layout); re-prepares the layers
    void set_split(const int g1[6]);
    // A CUDA graph of one bootstrap of `in` (members = 0: ordinary ciphertexts).  `out`
    // receives a buffer of the output's shape, rewritten by every Graph::launch; write the
    // next batch into `in` (same count and level) between launches.
    std::unique_ptr<Graph> capture(const Ciphertext &in, uint32_t members, Ciphertext &out) const;
    const BootstrapParams &params() const { return p_; }

   private:
    void slots_to_re_im(const Evaluator &ev, Ciphertext x, Ciphertext &re, Ciphertext &im) const;
    Ciphertext finish(const Evaluator &ev, const Ciphertext &re, const Ciphertext &im) const;

    Evaluator &ev_;
    BootstrapParams p_;
    std::vector<LinearTransform *> s2c_, c2s_;
    mutable std::vector<LinearTransform *> s2c_late_;  // SlotToCoeff after EvalMod (C2S-first)
    mutable uint32_t late_level_ = 0;
    mutable std::mutex late_mu_;
    std::vector<double> cheb_;
    double q0_ = 0, c_fin_ = 0;
    uint32_t top_ = 0;
};

// ---- one BERT encoder layer (layer.cpp; src/include/test/test_single_layer.cuh:422-2062)

struct BertLayerConfig {
    uint32_t hidden = 768, heads = 12, ffn = 3072;
    uint32_t num_X = 256, tokens = 128;  // inputs x tokens fill the N/2 slots (column packing)
    uint32_t input_num = 128;            // the softmax masks' band (softmax.cuh): valid tokens per input
    int softmax_iter = 13;               // inverse iterations of the softmax's sum
    int ln_newt = 3, ln_gold = 2;        // LayerNorm's inverse square root: 2 (newt + gold) + 8 levels
    double ln_var_scale = 64.0;          // see layernorm
    double w_scale = 1099511627776.0;    // 2^40: integer weights of the exact contractions
    uint32_t gelu_input_level = 13;      // GELU (6 levels) then the masked Final (2) and one to adjust
    uint32_t ffn_chunk = 256;            // Intermediate + GELU columns per pass (bounds the working set)
    uint32_t members = 0;                // shared-a group size of the bootstrap segments; 0 = ordinary
    uint32_t boot_batch = 16;            // ciphertexts per bootstrap call (1 = one per call)
};

// row-major [in][out] weight matrices and per-column vectors
struct BertLayerWeights {
    std::vector<double> Wq, Wk, Wv, Wo;  // [hidden][hidden]
    std::vector<double> bq, bk, bv, bo, ln1_gamma, ln1_beta, ln2_gamma, ln2_beta, bf;  // [hidden]
    std::vector<double> Wi, bi;  // [hidden][ffn], [ffn]
    std::vector<double> Wf;      // [ffn][hidden]
};

struct StageTime {
    std::string name;
    double seconds;
    size_t peak_bytes = 0;  // the context pool's high-water mark of device memory in use during the stage
};

// the steps of the attention's rotations (multiples of N/2 / tokens); generate their Galois keys
std::vector<int> bert_layer_rotation_steps(const BertLayerConfig &cfg, uint32_t slots);
// column o of Y plus b[o] on the slots marked 1 by mask (all slots when mask is empty)
Ciphertext add_column_bias(const Evaluator &ev, const Ciphertext &Y, const std::vector<double> &b,
                           const std::vector<int> &mask);
// x brought to the bootstrap's input level and scale, then bootstrapped in calls of `batch`
// ciphertexts (shared-a groups of `members`, a short last group padded; 0 = ordinary)
Ciphertext bootstrap_segment(const Evaluator &ev, const BatchBootstrapper &boot, const Ciphertext &x,
                             uint32_t members, uint32_t batch);
// the same, releasing x once it is at the input level (x is left empty): the segment's own
// working set then sits beside the small input batch instead of the whole-level one
Ciphertext bootstrap_segment(const Evaluator &ev, const BatchBootstrapper &boot, Ciphertext &&x, uint32_t members,
                             uint32_t batch);
// One layer on X (hidden columns at the bootstrap's output level and scale); the output has X's
// level and scale.  ev needs the relinearisation key, the Galois keys of the bootstrap (ordinary)
// or the shared-a keys of `members`, and the Galois keys of bert_layer_rotation_steps: either in
// ev.galois_keys or, with attention_keys, made from that key generator for the attention block
// and released after it (their time counts in the block).  times receives the 11 stages in the
// reference's names and order.
Ciphertext bert_layer(const Evaluator &ev, const BatchBootstrapper &boot, const Ciphertext &X,
                      const BertLayerWeights &w, const BertLayerConfig &cfg, const std::vector<int> &bias_vec,
                      std::vector<StageTime> *times = nullptr, KeyGenerator *attention_keys = nullptr);

// max |V w - layers(w)| / max |V w| of the slot-transform factorisation at n slots
// (a self-check of the planning code on random input)
double slot_transform_selfcheck(uint32_t log_slots);

// ------------------------------------------------------------------ serving loop

enum class JobKind : int { Rotate = 0, Matmul = 1, Bootstrap = 2 };

struct ServeResult {
    Ciphertext output;
    double t_submit = 0, t_start = 0, t_end = 0;  // seconds on the server's steady clock
    uint32_t batched_with = 1;                    // jobs that shared its launches (continuous batching)
    std::string error;                            // empty on success
};

struct ServeStats {
    size_t budget = 0, peak_admitted = 0;  // admission estimates, bytes
    uint32_t max_inflight = 0;             // most batches on the device at once
    uint64_t batches = 0, jobs = 0;        // launches groups run, jobs completed
};

// A request loop over one device: jobs (key-switch / rotation batches, ct-pt matmuls,
// shared-a or ordinary bootstraps) are admitted while their estimated device memory fits
// the HBM budget and a slot is free; each slot is a worker thread with its own stream and
// evaluator, so admitted batches overlap on the GPU; queued jobs of the same kind and
// shape join the batch a slot starts (continuous batching).  Keys and the bootstrapper's
// diagonals stay resident and are shared read-only.  Every result equals the job run
// alone: ciphertexts are independent units and shared-a groups never span two jobs.
class Server {
   public:
    Server(const Evaluator &base, const BatchBootstrapper *boot, const std::map<uint32_t, SharedAKeys> *shared,
           size_t hbm_budget, uint32_t slots, uint32_t max_merge = 64);
    ~Server();  // finishes the queued jobs, then stops the slots
    uint64_t submit_rotate(Ciphertext &&ct, int step);
    uint64_t submit_matmul(Ciphertext &&X, std::vector<int64_t> W, uint32_t n_out, double w_scale);
    uint64_t submit_bootstrap(Ciphertext &&ct, uint32_t members);
    ServeResult wait(uint64_t id);  // blocks until the job is done and hands its result over
    // while paused, slots start no new batch (queued jobs wait; running ones finish)
    void set_paused(bool paused);
    ServeStats stats() const;
    static double now();

   private:
    struct Job;
    struct Slot;
    uint64_t enqueue(std::unique_ptr<Job> j);
    size_t estimate(const Job &j) const;
    void worker(uint32_t slot);
    void run(Slot &s, std::vector<Job *> &batch);

    const Evaluator &base_;
    const BatchBootstrapper *boot_;
    const std::map<uint32_t, SharedAKeys> *shared_;
    size_t budget_;
    uint32_t max_merge_;
    struct State;
    std::unique_ptr<State> st_;
};

}  // namespace shmoai
