/* C ABI of the C++ host library (include/shmoai/host.hpp): key material, encryption,
 * the batched evaluator and S2C-first (shared-a) bootstrapping behind opaque handles,
 * for C callers and FFI bindings (ctypes in this repository's Python layer).
 *
 * Replaces the entry points the MOAI driver reaches through the reference's C++ classes:
 *   shm_host_*      moai::Encoder / Encryptor / Evaluator / Decryptor and key generation
 *                   (src/include/source/ckks_evaluator_parallel.cuh:13-598,
 *                   thirdparty/phantom-fhe/src/secretkey.cu:328-646);
 *   shm_host_*shared*  SharedAKeyGen, fmt_switch_forward / fmt_switch_backward, shared_a_rotate
 *                   (src/include/source/bootstrapping/FmtSwitch.cu:154-429, ShRotate.cu:54-257);
 *   shm_boot_*      BatchBootstrapper::{prepare, prepare_shared_keys,
 *                   bootstrap_ordinary_s2c_first, bootstrap_shared_a_s2c_first}
 *                   (src/include/source/bootstrapping/BatchBootstrap.cuh:470-819).
 * Status codes are those of include/shmoai_ckks.h; shm_host_last_error() explains the
 * last failure of the calling thread.  A shm_ct is a batch: ordinary ciphertexts
 * [count][size][L][N], or shared-a groups [count][members + 1][L][N] (shared = 1). */
#ifndef SHMOAI_HOST_H
#define SHMOAI_HOST_H
#include <stddef.h>
#include <stdint.h>

#include "shmoai_ckks.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct shm_host shm_host;
typedef struct shm_ct shm_ct;
typedef struct shm_boot shm_boot;
typedef struct shm_host_graph shm_host_graph;

const char *shm_host_last_error(void);

/* Context (n_primes = n_q + n_special, special primes last), secret key of Hamming weight
 * `hamming_weight`, deterministic in `seed`. */
int shm_host_create(shm_host **out, uint32_t log_n, const uint64_t *primes, uint32_t n_primes, uint32_t n_special,
                    int device, uint32_t hamming_weight, uint64_t seed);
int shm_host_create_from_bits(shm_host **out, uint32_t log_n, const int *bits, uint32_t n_primes,
                              uint32_t n_special, int device, uint32_t hamming_weight, uint64_t seed);
void shm_host_destroy(shm_host *h);
const shm_context *shm_host_context(const shm_host *h);
/* the n_q + n_special primes of the host's context */
int shm_host_primes(const shm_host *h, uint64_t *out);
int shm_host_synchronize(shm_host *h);
/* device bytes the host library holds now and at its peak (keys, ciphertexts, workspaces);
 * reset_peak != 0 restarts the peak from the current use */
int shm_host_device_memory(shm_host *h, size_t *in_use, size_t *peak, int reset_peak);

int shm_host_gen_relin_key(shm_host *h);
int shm_host_gen_galois_keys(shm_host *h, const uint32_t *elts, uint32_t n_elts);
/* auxiliary secrets, format key, backward keys and the Sh-Galois keys of `elts` for
 * shared-a groups of `members` */
int shm_host_gen_shared_keys(shm_host *h, uint32_t members, uint32_t hamming_weight, const uint32_t *elts,
                             uint32_t n_elts);
uint32_t shm_host_galois_elt(const shm_host *h, int step);

/* Encrypt `count` rows of n_values complex slot values (re, im: [count][n_values]) at L
 * primes and `scale`. */
int shm_host_encrypt(shm_host *h, const double *re, const double *im, uint32_t count, uint32_t n_values, uint32_t L,
                     double scale, shm_ct **out);
/* Public-key encryption (PhantomPublicKey::encrypt_asymmetric, secretkey.cu:15-217):
 * shm_host_gen_public_key makes pk = (e - a s, a) over QP from the host's secret
 * (gen_publickey, secretkey.cu:524-537) and a public-key encryptor whose samplers start at
 * `seed`; shm_host_encrypt_public then encrypts like shm_host_encrypt with u pk + (e0, e1)
 * brought down from QP to Q (the first L limbs kept) in place of the secret key. */
int shm_host_gen_public_key(shm_host *h, uint64_t seed);
int shm_host_encrypt_public(shm_host *h, const double *re, const double *im, uint32_t count, uint32_t n_values,
                            uint32_t L, double scale, shm_ct **out);
/* The MOAI packing (src/include/source/matrix_mul/Batch_encode_encrypt.cuh):
 * shm_host_batch_input replaces batch_input (:12-43): X [num_X][num_row][num_col] doubles ->
 * num_col ciphertexts, column i with slot num_X * k + j = X[j][k][i], encrypted with the
 * public key at L primes and `scale`.  shm_host_bias_vec replaces bias_vec (:45-56): out
 * [num_X * num_row] with slot j * num_X + i = 1 for j < lengths[i]. */
int shm_host_batch_input(shm_host *h, const double *X, uint32_t num_X, uint32_t num_row, uint32_t num_col,
                         double scale, uint32_t L, shm_ct **out);
int shm_host_bias_vec(const int *lengths, uint32_t num_X, uint32_t num_row, int *out);
/* Decrypt to [members in the batch][N/2] slot values (shared-a groups: member i of group
 * g is row g * members + i). */
int shm_host_decrypt(shm_host *h, const shm_ct *ct, double *re, double *im);

int shm_ct_from_host(shm_host *h, const uint64_t *data, uint32_t count, uint32_t size, uint32_t L, double scale,
                     int shared, shm_ct **out);
int shm_ct_to_host(shm_host *h, const shm_ct *ct, uint64_t *data);
/* Integer coefficients [N] of one slot vector (re, im: n_values host doubles) at `scale`: by
 * the device encoder (on_host = 0, shm_encode) or by the host's FFT restatement (on_host = 1,
 * shmoai::Encoder::encode_float + round half to even); the two are equal bit for bit. */
int shm_host_encode(shm_host *h, const double *re, const double *im, uint32_t n_values, double scale,
                    int64_t *coeffs, int on_host);
/* overwrite the residues of an existing batch from host words laid out as shm_ct_to_host
 * writes them (same count, size and level) */
int shm_ct_write(shm_host *h, shm_ct *ct, const uint64_t *data);
int shm_ct_info(const shm_ct *ct, uint32_t *count, uint32_t *size, uint32_t *L, double *scale, int *shared);
/* a device copy of ciphertexts [first, first + count) of a batch */
int shm_host_slice(shm_host *h, const shm_ct *ct, uint32_t first, uint32_t count, shm_ct **out);
const uint64_t *shm_ct_device_data(const shm_ct *ct);
void shm_ct_destroy(shm_ct *ct);

int shm_host_add(shm_host *h, const shm_ct *a, const shm_ct *b, shm_ct **out);
int shm_host_sub(shm_host *h, const shm_ct *a, const shm_ct *b, shm_ct **out);
/* multiply + relinearise + rescale */
int shm_host_multiply(shm_host *h, const shm_ct *a, const shm_ct *b, shm_ct **out);
int shm_host_rescale(shm_host *h, const shm_ct *a, shm_ct **out);
int shm_host_multiply_const(shm_host *h, const shm_ct *a, double value, shm_ct **out);
int shm_host_rotate(shm_host *h, const shm_ct *a, int step, shm_ct **out);
int shm_host_conjugate(shm_host *h, const shm_ct *a, shm_ct **out);
int shm_host_multiply_i(shm_host *h, const shm_ct *a, int sign, shm_ct **out);
/* rotation-free ct-pt matmul + rescale: W host [n_in][n_out] encoded integer weights
 * (|W| < 2^40) at w_scale; tensor_cores = 0 runs the CUDA-core kernel (the plain path) */
int shm_host_ctpt_matmul(shm_host *h, const shm_ct *X, const int64_t *W, uint32_t n_out, double w_scale,
                         int tensor_cores, shm_ct **out);
/* the masked projection (ct_pt_matrix_mul_wo_pre_w_mask, Ct_pt_matrix_mul.cuh:846-986):
 * mask [N/2] slot values multiply every output of the ct-pt matmul; one mask plaintext, two
 * levels (the reference: n_in * n_out masked-weight plaintexts, one level) */
int shm_host_ctpt_matmul_masked(shm_host *h, const shm_ct *X, const int64_t *W, uint32_t n_out, double w_scale,
                                const double *mask, int tensor_cores, shm_ct **out);
/* Polynomial operators (the BERT layer's non-linear functions, src/include/source/non_linear_func/):
 * sum_k coeffs[k] T_k(u), u = (2 x - hi - lo) / (hi - lo), on every slot of an ordinary batch,
 * output at the input's scale; and GELU by gelu_cheb's degree-24 series on [-19.5, 12.5]
 * (non_linear_func/gelu_other.cuh:258-300).  They consume 1 + depth(series) levels (degree 24:
 * 6, where gelu_cheb takes 7); SHM_EINVAL when the input has too few. */
int shm_host_chebyshev(shm_host *h, const shm_ct *a, const double *coeffs, uint32_t n_coeffs, double lo, double hi,
                       shm_ct **out);
int shm_host_gelu(shm_host *h, const shm_ct *a, shm_ct **out);
/* the softmax's building blocks (non_linear_func/softmax.cuh:23-118): exp(x) as (1 + x/128)^128
 * (8 levels), and 1/x for x in (0, 2) as prod_{i <= iter} (1 + (1 - x)^(2^i)) (iter + 1 levels) */
int shm_host_exp(shm_host *h, const shm_ct *a, shm_ct **out);
int shm_host_inverse(shm_host *h, const shm_ct *a, uint32_t iter, shm_ct **out);
/* 1/sqrt(x) for LayerNorm (invert_sqrt, non_linear_func/layernorm.cuh:708-897): the first
 * guess -1.29054537e-4 x + 0.129054537, d_newt Newton and d_gold Goldschmidt steps */
int shm_host_inv_sqrt(shm_host *h, const shm_ct *a, uint32_t d_newt, uint32_t d_gold, shm_ct **out);
/* LayerNorm over the hidden columns of the column packing, one column per ciphertext of the
 * batch `a` (layernorm, non_linear_func/layernorm.cuh:899-): gamma[i] (x_i - mean) / sqrt(var)
 * + beta[i] with the inverse square root above (gamma, beta: one value per ciphertext);
 * 2 (d_newt + d_gold) + 8 levels */
int shm_host_layernorm(shm_host *h, const shm_ct *a, const double *gamma, const double *beta, uint32_t d_newt,
                       uint32_t d_gold, shm_ct **out);
/* softmax over the ciphertexts of a batch (softmax, non_linear_func/softmax.cuh:119-, without
 * the attention layout's masks): e_i / sum_j e_j, e_i = exp(x_i - shift) as above, the sum's
 * inverse by shm_host_inverse on sum_scale * sum_j e_j (the caller keeps it in (0, 2));
 * iter + 12 levels */
int shm_host_softmax(shm_host *h, const shm_ct *a, double shift, double sum_scale, uint32_t iter, shm_ct **out);
/* the attention block's softmax with its masks (softmax, non_linear_func/softmax.cuh:119-):
 * bias_vec has one 0/1 entry per slot (N/2), input_num is the reference's band of diagonals;
 * iter + 10 levels */
int shm_host_softmax_attention(shm_host *h, const shm_ct *a, const int *bias_vec, int input_num, uint32_t iter,
                               shm_ct **out);
/* attention's ct-ct product in the column packing (ct_ct_matrix_mul_colpacking,
 * matrix_mul/Ct_ct_matrix_mul.cuh:10-120): X and W batches of the same count, output batch of
 * `rows` ciphertexts out_i = sum_j X_j * rot(W_j, i * num_batch), relinearised and rescaled;
 * the Galois keys of the steps i * num_batch must have been generated */
int shm_host_ct_ct_matmul(shm_host *h, const shm_ct *X, const shm_ct *W, uint32_t rows, uint32_t num_batch,
                          shm_ct **out);
/* the diagonal-packed ct-ct product (ct_ct_matrix_mul_diagpacking, Ct_ct_matrix_mul.cuh:182-):
 * X holds the diagonals, W the columns; output batch of W.count ciphertexts (1 level) */
int shm_host_ct_ct_matmul_diag(shm_host *h, const shm_ct *X, const shm_ct *W, uint32_t num_batch, shm_ct **out);
/* a CUDA graph of shm_host_chebyshev (coeffs = NULL: GELU) on `in`; *out is rewritten by every
 * shm_host_graph_launch; write the next batch into `in` with shm_ct_write between launches */
int shm_host_chebyshev_capture(shm_host *h, const shm_ct *in, const double *coeffs, uint32_t n_coeffs, double lo,
                               double hi, shm_ct **out, shm_host_graph **graph);
int shm_host_to_shared(shm_host *h, const shm_ct *a, uint32_t members, shm_ct **out);
int shm_host_from_shared(shm_host *h, const shm_ct *a, shm_ct **out);

/* Bootstrapper at the host's parameters (scale Delta, input at `input_level` primes);
 * prepares the slot-transform diagonals and the EvalMod polynomial. */
int shm_boot_create(shm_host *h, double scale, uint32_t input_level, shm_boot **out);
void shm_boot_destroy(shm_boot *b);
/* the Galois elements its rotations need (n_out set; at most `cap` written) */
int shm_boot_galois_elts(const shm_boot *b, uint32_t *out, uint32_t cap, uint32_t *n_out);
/* bootstrap a batch at input_level primes; members = 0: ordinary ciphertexts,
 * members = n: shared-a groups of n consecutive ciphertexts (keys from
 * shm_host_gen_shared_keys) */
int shm_boot_run(shm_boot *b, const shm_ct *in, uint32_t members, shm_ct **out);
/* The original per-ciphertext C2S-first bootstrap (Bootstrapper::bootstrap_3,
 * Bootstrapper.cu:3606-3627, 3889-3903): ordinary ciphertexts at one prime (or brought there
 * at scale Delta), ModRaise, CoeffToSlot, EvalMod, SlotToCoeff; the first call encodes the
 * late SlotToCoeff diagonals. */
int shm_boot_run_c2s_first(shm_boot *b, const shm_ct *in, shm_ct **out);
/* One BERT encoder layer (src/include/test/test_single_layer.cuh:422-2062) on X: hidden
 * columns in the column packing at the bootstrap's output level and scale.
 * dims: hidden, heads, ffn, num_X, tokens, input_num, softmax_iter, ln_newt, ln_gold,
 *       gelu_input_level, ffn_chunk, members (shared-a group size of the bootstrap segments,
 *       0 = ordinary), boot_batch (ciphertexts per bootstrap call);
 * reals: w_scale (integer weights of the contractions), ln_var_scale;
 * weights: Wq [d][d], bq [d], Wk, bk, Wv, bv, Wo, bo, ln1_gamma [d], ln1_beta [d],
 *          Wi [d][ffn], bi [ffn], Wf [ffn][d], bf [d], ln2_gamma, ln2_beta, concatenated;
 * bias_vec: N/2 ints (1 = valid token slot).  The host needs the relinearisation key, the Galois
 * keys of the attention's rotation steps (multiples of N/2 / tokens) and, for members = 0, of the
 * bootstrap, else the shared-a keys of groups of `members`.  stage_seconds receives 22 values:
 * the wall times of Attention Block, SelfOutput, 1st Bootstrapping, LayerNorm1, 2nd
 * Bootstrapping, Intermediate Linear, GELU, Final Linear, 3rd Bootstrapping, LayerNorm2, 4th
 * Bootstrapping, then the device memory high-water mark (GiB, the context pool) of each stage. */
int shm_boot_bert_layer(shm_boot *b, const shm_ct *X, const uint32_t *dims, const double *reals, const double *weights,
                        const int *bias_vec, shm_ct **out, double *stage_seconds);
/* autotuning for batches of `count` (shmoai::BatchBootstrapper::tune): NTT tile, Sh-Rot
 * inner-product chunk, BSGS split per slot-transform layer; call before generating the
 * Galois / Sh-Galois keys (shm_boot_galois_elts changes with the split).  Writes a JSON
 * array of {"knob", "candidates", "ms", "chosen"} into `json` (NUL-terminated, truncated at
 * cap); *needed (may be NULL) = the full length + 1. */
int shm_boot_tune(shm_boot *b, uint32_t count, uint32_t members, char *json, size_t cap, size_t *needed);
/* the BSGS baby-step counts of the six slot-transform layers (S2C 0-2, C2S 3-5; 0 = default):
 * read the tuned split, or set a stored one (re-prepares the layers) */
int shm_boot_get_split(const shm_boot *b, int *g1);
int shm_boot_set_split(shm_boot *b, const int *g1);

/* CUDA graph of one shm_boot_run of `in` (shmoai::BatchBootstrapper::capture): the
 * bootstrap runs once on the host's stream and once on a private stream before it is
 * recorded; *out receives the output ciphertext, which every shm_host_graph_launch
 * rewrites.  Put the next batch into `in` with shm_ct_write between launches; `in` must
 * outlive the graph. */
int shm_boot_capture(shm_boot *b, const shm_ct *in, uint32_t members, shm_ct **out, shm_host_graph **graph);
/* replay on the host's stream */
int shm_host_graph_launch(shm_host_graph *g);
uint64_t shm_host_graph_kernels(const shm_host_graph *g);
void shm_host_graph_destroy(shm_host_graph *g);

/* self-check of the slot-transform factorisation at 2^log_slots slots (max error) */
double shm_slot_transform_selfcheck(uint32_t log_slots);

/* ---- binary records (include/shmoai/wire.hpp): an 80-byte header naming the kind, ring,
 * prime-chain digest, shape and scale, the payload words, then a digest of header and payload.
 * Loading checks the header against the host's context, every residue against its prime
 * and the digest; a failure returns SHM_EINVAL and builds nothing.
 * Ciphertext batches go to and from caller memory: shm_ct_serialized_bytes gives the size
 * of the record, shm_ct_serialize writes it (cap must hold it), shm_ct_deserialize reads
 * exactly one record of `len` bytes. */
int shm_ct_serialized_bytes(shm_host *h, const shm_ct *ct, size_t *bytes);
int shm_ct_serialize(shm_host *h, const shm_ct *ct, void *buf, size_t cap);
int shm_ct_deserialize(shm_host *h, const void *buf, size_t len, shm_ct **out);
/* The host's keys to and from a file: the secrets (with_secrets != 0: the secret and the
 * auxiliary secrets of the last shm_host_gen_shared_keys), the relinearisation key, the
 * Galois keys and every shared-a key set.  Loading replaces what the file holds and keeps
 * the rest (a Galois key of another element stays). */
int shm_host_save_keys(shm_host *h, const char *path, int with_secrets);
int shm_host_load_keys(shm_host *h, const char *path);
/* The secret as the reference's text file: Q*P*N decimal residues in NTT form, limb-major,
 * one per line (PhantomSecretKey::load_secret_key,
 * thirdparty/phantom-fhe/include/secretkey.h:290-307).  Import replaces the host's secret
 * (keys generated afterwards use it; existing keys are kept); the residues must be one
 * small integer polynomial. */
int shm_host_import_secret_text(shm_host *h, const char *path);
int shm_host_export_secret_text(shm_host *h, const char *path);
/* Install an evaluation key from host words laid out as the reference's key digits,
 * [dnum][2][QP][N] (b then a, NTT form; PhantomRelinKey / PhantomGaloisKey,
 * thirdparty/phantom-fhe/src/secretkey.cu:328-373): kind 0 = relinearisation key,
 * kind 1 = Galois key of element `elt`.  n_words must be dnum * 2 * QP * N. */
#define SHM_KEY_RELIN 0
#define SHM_KEY_GALOIS 1
int shm_host_import_key(shm_host *h, int kind, uint32_t elt, const uint64_t *words, size_t n_words);

/* ---- serving loop (shmoai::Server): jobs admitted by an HBM budget onto `slots`
 * concurrent streams, queued jobs of the same kind and shape batched together.  Submit
 * calls take ownership of the ciphertext handle (it is destroyed, the caller must not use
 * it again); results come back through shm_server_wait.  `boot` may be NULL (no
 * bootstrap jobs).  The host, the bootstrapper and the keys must outlive the server. */
typedef struct shm_server shm_server;
int shm_server_create(shm_host *h, shm_boot *boot, size_t hbm_budget_bytes, uint32_t slots, uint32_t max_merge,
                      shm_server **out);
void shm_server_destroy(shm_server *s); /* finishes queued jobs first */
int shm_server_submit_rotate(shm_server *s, shm_ct *ct, int step, uint64_t *job);
/* W: host [n_in][n_out] encoded integer weights (|W| < 2^40), output rescaled once */
int shm_server_submit_matmul(shm_server *s, shm_ct *X, const int64_t *W, uint32_t n_out, double w_scale,
                             uint64_t *job);
int shm_server_submit_bootstrap(shm_server *s, shm_ct *ct, uint32_t members, uint64_t *job);
/* blocks until `job` is done; times = {submit, start, end} in seconds (steady clock);
 * batched_with = jobs that shared its launches; the job's error is returned as a status */
int shm_server_wait(shm_server *s, uint64_t job, shm_ct **out, double *times, uint32_t *batched_with);
/* paused = 1: slots start no new batch until resumed (queued jobs wait, running ones finish) */
int shm_server_set_paused(shm_server *s, int paused);
int shm_server_stats(const shm_server *s, size_t *budget, size_t *peak_admitted, uint32_t *max_inflight,
                     uint64_t *batches, uint64_t *jobs);

#ifdef __cplusplus
}
#endif
#endif /* SHMOAI_HOST_H */
