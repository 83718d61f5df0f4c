// Internal interface of the CKKS core: the device-resident context and the
// kernel launchers.  The public surface is the C ABI in include/shmoai_ckks.h.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "modarith.cuh"
#include "ntt.cuh"

namespace shm {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Number of kernels this library has launched (reported by shm_kernel_launches).
extern std::atomic<unsigned long long> g_launches;
#define SHM_LAUNCHED(k) ::shm::g_launches.fetch_add((k), std::memory_order_relaxed)

#define SHM_CUDA(call)                                                                                       \
    do {                                                                                                     \
        cudaError_t e_ = (call);                                                                             \
        if (e_ != cudaSuccess)                                                                               \
            throw ::shm::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " at " __FILE__ ":" + \
                                   std::to_string(__LINE__));                                                \
    } while (0)

// Per-level constants of hybrid key switching with L data limbs.
struct LevelKS {
    uint32_t L = 0, beta = 0;
    uint64_t *modup_scale = nullptr;  // [L][4]: N^-1 * qhat_i^-1 (digit-relative), for the INTT's last stage
    uint64_t *modup_conv = nullptr;   // [beta][L+np][alpha]: qhat_i mod t_j (0 on the digit's own rows)
    // ModDown by S = q_{L-1} P (relinearisation and rescale in one; L >= 2): s_0 = q_{L-1},
    // s_{1+k} = p_k
    uint64_t *rr_scale = nullptr;  // [np + 1][4]: N^-1 * (S / s_k)^-1 mod s_k, for the INTT's last stage
    uint64_t *rr_conv = nullptr;   // [L - 1][np + 1]: (S / s_k) mod q_j
    uint64_t *rr_sinv = nullptr;   // [L - 1][2]: S^-1 mod q_j and its Shoup companion
    uint64_t *rr_vs = nullptr;     // [L - 1][16]: (v S) mod q_j for v < 16 (exact conversion)
    double *rr_inv_s = nullptr;    // [np + 1]: 1 / s_k rounded to double
};

// the slot that an NTT-domain automorphism X -> X^elt moves to slot k (N = 2^log_n):
// 2 brv(perm) + 1 = (2 brv(k) + 1) elt mod 2N, brv the log_n-bit reversal
__host__ __device__ __forceinline__ uint32_t galois_index(uint32_t k, uint32_t elt, uint32_t log_n) {
#ifdef __CUDA_ARCH__
    const uint32_t bk = __brev(k) >> (32 - log_n);
#else
    uint32_t bk = 0;
    for (uint32_t i = 0; i < log_n; i++) bk |= ((k >> i) & 1u) << (log_n - 1 - i);
#endif
    const uint32_t e = (uint32_t)(((uint64_t)(2 * bk + 1) * elt) & ((2ull << log_n) - 1));
    const uint32_t h = (e - 1) >> 1;
#ifdef __CUDA_ARCH__
    return __brev(h) >> (32 - log_n);
#else
    uint32_t r = 0;
    for (uint32_t i = 0; i < log_n; i++) r |= ((h >> i) & 1u) << (log_n - 1 - i);
    return r;
#endif
}

struct Context {
    int device = 0;
    uint32_t log_n = 0, n = 0, nq = 0, np = 0, dnum = 0;
    std::vector<uint64_t> primes;       // nq + np
    bool s52 = false;                   // every prime below kS52PrimeLimit (Acc<true> kernels)
    int ntt_variant = 0;                // index into kNttVariants (set by the autotuner)
    int ntt_families = 0;               // the NTT instantiation for the primes' butterfly families (kFam*)
    uint32_t ip_chunk_bytes = 32768;    // shared memory per Sh-Rot inner-product block (autotuned)
    std::vector<PrimeConst> h_pc;       // host copy
    PrimeConst *pc = nullptr;           // [QP]
    uint64_t *tw = nullptr;             // [QP][4][N]
    double *twq = nullptr;              // [QP][3][N]: the forward and inverse twiddles over q, and the forward twiddles, as doubles
    uint64_t *inv_scale_plain = nullptr;  // [QP][4]: N^-1 for a plain INTT, indexed by prime
    uint64_t *moddown_scale = nullptr;  // [np][4]: N^-1 * phat_k^-1
    uint64_t *moddown_conv = nullptr;   // [nq][np]: phat_k mod q_j
    uint64_t *p_inv = nullptr;          // [nq][2]: P^-1 mod q_j and Shoup companion
    uint64_t *p_mod = nullptr;          // [nq][2]: P mod q_j and Shoup companion (extended basis)
    std::vector<uint64_t> h_p_mod;      // host copy
    uint64_t *rescale_inv = nullptr;    // [nq][nq][2]: q_{L-1}^-1 mod q_j (row L-1), Shoup
    std::vector<LevelKS> ks;            // index L (1..nq)
    std::map<uint32_t, uint32_t *> galois_perm;  // elt -> [N] permutation
    std::map<uint32_t, std::vector<void *>> ext_consts;  // L -> exact Ql->P extension tables (shared.cu)
    std::mutex mu;

    // internal arena for calls that pass no workspace
    void *arena = nullptr;
    size_t arena_bytes = 0;

    // stream-ordered allocation pool of shm_malloc / shm_free (created on first use);
    // freed blocks stay in the pool for reuse
    cudaMemPool_t pool = nullptr;

    ~Context();
    const uint32_t *perm(uint32_t elt);
    void *workspace(size_t bytes);
    cudaMemPool_t mempool();
};

Context *create_context(uint32_t log_n, const std::vector<uint64_t> &primes, uint32_t nq, uint32_t np, int device);

// ---------------- launchers (all asynchronous on `st`) ----------------
// NTT of `rows` limbs of N words; limb r uses prime map.prime[r % slots] (255 = skip).
void ntt_forward(const Context &c, uint64_t *data, uint32_t rows, uint32_t slots, const LimbMap &map,
                 cudaStream_t st);
// Inverse NTT; `scale` is [slots - scale_base][4] (c, c', c*psi^-(N/2), shoup), or nullptr
// for the plain N^-1 of each limb's prime.
void ntt_inverse(const Context &c, uint64_t *data, uint32_t rows, uint32_t slots, const LimbMap &map,
                 const uint64_t *scale, cudaStream_t st, uint32_t scale_base = 0);

LimbMap q_map(uint32_t L);
// forward NTT of the rescale's spread limbs fused with the spread and the combine (RescaleIO);
// t: [n_polys][L-1][N] scratch between the two phases
void ntt_forward_rescale(const Context &c, const RescaleIO &io, uint64_t *t, uint32_t n_polys, uint32_t L,
                         cudaStream_t st);
// ModDown's conversion, forward NTT and combine in one launch pair (ModDownIO); delta:
// [n_polys][L][N] scratch between the two phases
// ModUp's base conversion, forward NTT and the digit copies in one launch pair (ModUpIO): up
// [n_cts][beta][LP][N] with map = the prime of every converted row, 255 on the digits' own rows
void ntt_forward_modup(const Context &c, const ModUpIO &mu, uint64_t *up, uint32_t n_cts, uint32_t beta,
                       const LimbMap &map, cudaStream_t st);
void ntt_forward_moddown(const Context &c, const ModDownIO &md, uint64_t *delta, uint32_t n_polys, uint32_t L,
                         cudaStream_t st);

enum class EwOp { Add, Sub, Negate, MulPlain };
void elementwise(const Context &c, EwOp op, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys,
                 uint32_t L, uint32_t b_polys, cudaStream_t st);
void tensor(const Context &c, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_cts, uint32_t L,
            cudaStream_t st);
void add_sizes(const Context &c, const uint64_t *a, uint32_t sa, const uint64_t *b, uint32_t sb, uint64_t *out,
               uint32_t n_cts, uint32_t L, cudaStream_t st);
void apply_galois(const Context &c, const uint64_t *in, uint64_t *out, uint32_t rows, uint32_t elt, cudaStream_t st);
void rescale(const Context &c, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t *ws,
             cudaStream_t st);
size_t rescale_ws_words(const Context &c, uint32_t n_polys, uint32_t L);

// Hybrid key switch of n_cts polynomials d (NTT form, [n_cts][L][N], stride d_stride words)
// with key [dnum][2][QP][N].  out0/out1 ([n_cts][L][N], stride out_stride):
//   out0 = add0 + cx0, out1 = add1 + cx1 (add0/add1 may be null meaning zero).
struct KsOutput {
    uint64_t *out0, *out1;
    const uint64_t *add0, *add1;
    size_t stride;                // words between consecutive ciphertexts for out/add
    const uint32_t *add0_perm;    // if set, add0 is read at add0_perm[k] (an automorphism)
};
void keyswitch(const Context &c, const uint64_t *d, size_t d_stride, uint32_t n_cts, uint32_t L, const uint64_t *key,
               const KsOutput &o, uint64_t *ws, cudaStream_t st);
size_t keyswitch_ws_words(const Context &c, uint32_t n_cts, uint32_t L);
// Relinearisation and rescale of n_cts size-3 ciphertexts ct3 [n_cts][3][L][N] in one
// ModDown by S = q_{L-1} P with an exact conversion: out [n_cts][2][L-1][N] =
// floor((P c_h + ks_h) / S), which equals relinearize-then-rescale unless that sum lies
// within n_p + 1 of a multiple of q_{L-1} P; workspace keyswitch_ws_words(c, n_cts, L).
void relin_rescale(const Context &c, const uint64_t *ct3, uint32_t n_cts, uint32_t L, const uint64_t *key,
                   uint64_t *out, uint64_t *ws, cudaStream_t st);
// Hoisted automorphisms: one ModUp of the c1 of n_cts ciphertexts `ct` ([n_cts][2][L][N]),
// then per element e: outs[e] = (sigma_e(c0) + cx0, cx1) with keys[e].
void apply_galois_hoisted(const Context &c, const uint64_t *ct, uint32_t n_cts, uint32_t L, uint32_t n_elts,
                          const uint32_t *elts, const uint64_t *const *keys, uint64_t *const *outs, uint64_t *ws,
                          cudaStream_t st);
size_t hoisted_ws_words(const Context &c, uint32_t n_cts, uint32_t L);

// per-limb scalars passed by value (residue and Shoup companion per limb)
struct ScalarTab {
    uint64_t v[64], shoup[64];
};
constexpr int kMaxAccTerms = 32;
struct PtrTab {
    const uint64_t *p[kMaxAccTerms];
};
// out[ct] (+)= sum_{t < k} A_t[ct a_step] x B_t[ct b_step] (size-3 tensor products; k <= kMaxAccTerms,
// bounded by the caller so that 2k products stay below every limb's Barrett bound)
void tensor_accumulate(const Context &c, const PtrTab &A, const PtrTab &B, uint32_t k, uint32_t a_step,
                       uint32_t b_step, uint64_t *out, uint32_t n_cts, uint32_t L, bool accumulate, cudaStream_t st);
void mul_scalar(const Context &c, const uint64_t *a, uint64_t *out, const ScalarTab &s, uint32_t n_polys, uint32_t L,
                cudaStream_t st);
void add_scalar(const Context &c, const uint64_t *a, uint64_t *out, const ScalarTab &s, uint32_t n_cts, uint32_t L,
                cudaStream_t st);
// rows of L limbs (limb l -> prime l), or with ext the extended basis (rows of L + np limbs)
void mul_plain_acc(const Context &c, const PtrTab &X, const PtrTab &P, uint32_t k, uint64_t *out, uint32_t n_polys,
                   uint32_t L, bool accumulate, cudaStream_t st, bool ext = false);
// sum_t w_t X_t + w0 (c0 only) over size-2 ciphertexts; weights passed by value
constexpr int kMaxLinTerms = 8;
struct LinTerms {
    const uint64_t *x[kMaxLinTerms];
    uint32_t levels[kMaxLinTerms];
    uint64_t w[kMaxLinTerms][64], ws[kMaxLinTerms][64];  // residue and Shoup companion per limb
    uint64_t w0[64];
    uint32_t k;
    int has_w0;
};
void linear_combination(const Context &c, const LinTerms &t, uint64_t *out, uint32_t n_cts, uint32_t L,
                        cudaStream_t st);
// one-limb polynomials (mod q0, NTT form) -> L-limb centred lift (NTT form); ws: n_polys * N words
void modraise(const Context &c, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t *ws,
              cudaStream_t st);

void ctpt_matmul(const Context &c, const uint64_t *X, const int64_t *W, uint64_t *Y, uint32_t n_in, uint32_t n_out,
                 uint32_t L, uint64_t *ws, cudaStream_t st);
void ctpt_matmul_cuda_core(const Context &c, const uint64_t *X, const int64_t *W, uint64_t *Y, uint32_t n_in,
                           uint32_t n_out, uint32_t L, cudaStream_t st);
size_t ctpt_tc_ws_bytes(const Context &c, uint32_t n_in, uint32_t n_out, uint32_t L);

// canonical-embedding encode / decode in FP64 (encode.cu); encode returns false when a
// coefficient reaches 2^62
size_t encode_ws_bytes(const Context &c, uint32_t n_pts);
bool encode(const Context &c, const double *re, const double *im, uint32_t n_pts, uint32_t n_values, double scale,
            int64_t *coeffs, void *ws, cudaStream_t st);
void decode(const Context &c, const double *coeffs, uint32_t n_pts, double scale, double *re, double *im, void *ws,
            cudaStream_t st);
void release_encode_tables(const Context &c);

// counter-based samplers and the signed lift (sampling.cu)
void sample_uniform(const Context &c, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t seed, cudaStream_t st);
void sample_cbd(const Context &c, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t seed, cudaStream_t st);
void lift_signed(const Context &c, const int64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L, cudaStream_t st);

// ModUp of n_cts polynomials d (stride d_stride words) into up [n_cts][beta][LP][N]; x: [n_cts][L][N] scratch
void modup_into(const Context &c, const uint64_t *d, size_t d_stride, uint32_t n_cts, uint32_t L, uint64_t *x,
                uint64_t *up, cudaStream_t st);

// shared-a batches [n_groups][n + 1][L][N] = (b_0 .. b_{n-1}, a) (shared.cu)
size_t shared_rotate_ws_words(const Context &c, uint32_t n_groups, uint32_t n, uint32_t L);
void shared_rotate_hoisted(const Context &c, const uint64_t *sh, uint32_t n_groups, uint32_t n, uint32_t L,
                           uint32_t n_elts, const uint32_t *elts, const uint64_t *const *keys, uint64_t *const *outs,
                           uint64_t *ws, cudaStream_t st);
size_t fmt_forward_ws_words(const Context &c, uint32_t n_groups, uint32_t n, uint32_t L);
void fmt_forward(const Context &c, const uint64_t *cts, uint32_t n_groups, uint32_t n, uint32_t L,
                 const uint64_t *key, uint64_t *out, uint64_t *ws, cudaStream_t st);
size_t fmt_backward_ws_words(const Context &c, uint32_t n_groups, uint32_t n, uint32_t L);
void fmt_backward(const Context &c, const uint64_t *sh, uint32_t n_groups, uint32_t n, uint32_t L,
                  const uint64_t *const *keys, uint64_t *out, uint64_t *ws, cudaStream_t st);
// max_l1 = max over outputs o of sum_i |W_io| (it sizes the residue system)
void ctpt_matmul_tc(const Context &c, const uint64_t *X, const int64_t *W, uint64_t *Y, uint32_t n_in, uint32_t n_out,
                    uint32_t L, void *ws, uint64_t max_l1, cudaStream_t st);
int ctpt_tc_error(void *ws, cudaStream_t st);
size_t ctpt_ws_words(const Context &c, uint32_t n_in, uint32_t n_out, uint32_t L);
// ---- the extended basis QlP: a polynomial at level L has L + np limbs, the Q limbs 0..L-1
// (primes q_0 .. q_{L-1}) then the special primes p_0 .. p_{np-1} (shared.cu)
LimbMap ext_map(uint32_t L, const Context &c);
void extend(const Context &c, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L, cudaStream_t st);
void add_ext(const Context &c, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys, uint32_t L,
             cudaStream_t st);
size_t moddown_ext_ws_words(const Context &c, uint32_t n_polys, uint32_t L);
void moddown_ext(const Context &c, uint64_t *ext, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t *ws,
                 cudaStream_t st);
size_t shared_rotate_ext_ws_words(const Context &c, uint32_t n_groups, uint32_t n, uint32_t L);
void shared_rotate_ext(const Context &c, const uint64_t *in, bool in_ext, uint32_t n_groups, uint32_t n, uint32_t L,
                       uint32_t n_elts, const uint32_t *elts, const uint64_t *const *keys, uint64_t *const *outs,
                       uint64_t *ws, cudaStream_t st);
void lift_signed_ext(const Context &c, const int64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
                     cudaStream_t st);

// acc [n_cts][H][LP][N] = inner products of up [n_cts][beta][LP][N] with key [beta][H][QP][N]
void ip_multi(const Context &c, const uint64_t *up, const uint64_t *key, uint64_t *acc, uint32_t n_cts, uint32_t L,
              uint32_t beta, uint32_t H, const uint32_t *perm, cudaStream_t st);

// autotuning (tune.cu): time the candidates of one knob, keep the fastest in the context
constexpr uint32_t kIpChunkCandidates[] = {16384, 32768, 65536, 98304};
uint32_t tune_ntt_tile(Context &c, uint32_t rows, std::vector<float> &ms);
uint32_t tune_ip_chunk(Context &c, uint32_t groups, uint32_t L, uint32_t members, std::vector<float> &ms);

}  // namespace shm
