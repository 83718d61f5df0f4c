/*
 * shmoai_ckks.h -- C ABI of the B200 CKKS evaluation core.
 *
 * Drop-in boundary for ShMOAI's evaluator hot path.  Each entry point replaces
 * the reference operation cited beside it (paths are inside the ShMOAI tree);
 * results are bit-identical to the reference's for the same primes, keys and
 * inputs.
 *
 * Conventions
 *  - All ring data is uint64 residues in DEVICE memory, in NTT form unless a
 *    function says otherwise.  A polynomial at level L is [L][N] (limb i under
 *    prime i of the chain); a ciphertext is [2][L][N]; batches of ciphertexts
 *    are contiguous [n_cts][2][L][N].  This is the reference's own layout
 *    (thirdparty/phantom-fhe/include/ciphertext.h:274-282).
 *  - Key-switching keys are [dnum][2][nq+np][N]: per digit the "b" half
 *    (added into c0) followed by the "a" half (secretkey.cu:328-373 layout).
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).  Every call is
 *    asynchronous on that stream.
 *  - `workspace` / `workspace_bytes`: device scratch owned by the caller, at
 *    least shm_*_workspace_bytes(); pass NULL to use the context's internal
 *    arena (grown on demand; serialise such calls per context).
 *  - Every function returns SHM_OK or a negative SHM_E* code and never throws;
 *    shm_last_error() gives the message of the calling thread's last failure.
 */
#ifndef SHMOAI_CKKS_H
#define SHMOAI_CKKS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SHM_OK 0
#define SHM_EINVAL -1   /* bad argument (level, size, shape) */
#define SHM_ECUDA -2    /* CUDA runtime error */
#define SHM_ENOMEM -3   /* device allocation failed */
#define SHM_EINTERNAL -4

typedef struct shm_context shm_context;

/* Context over a prime chain given by bit sizes: n_q ciphertext primes then
 * n_p special primes, generated exactly like CoeffModulus::Create
 * (thirdparty/phantom-fhe/src/modulus.cu:79-110).  Replaces PhantomContext(parms)
 * (thirdparty/phantom-fhe/src/context.cu:141-238).  log_n in {12, 16}. */
int shm_context_create(shm_context **out, uint32_t log_n, const int *bits, uint32_t n_q, uint32_t n_p, int device);
/* Same with explicit primes (n_q + n_p values, each 1 mod 2N, < 2^61). */
int shm_context_create_from_primes(shm_context **out, uint32_t log_n, const uint64_t *primes, uint32_t n_q,
                                   uint32_t n_p, int device);
void shm_context_destroy(shm_context *ctx);
/* log_n, n_q, n_p, dnum = n_q / n_p (secretkey.cu:341) */
int shm_context_info(const shm_context *ctx, uint32_t *log_n, uint32_t *n_q, uint32_t *n_p, uint32_t *dnum);
int shm_context_primes(const shm_context *ctx, uint64_t *out);
const char *shm_last_error(void);
/* Total kernels launched by this library in this process (no reference
 * counterpart: instrumentation for the benchmark's launch count). */
uint64_t shm_kernel_launches(void);

/* Forward / inverse negacyclic NTT of n_polys polynomials of L limbs, in place.
 * Replaces nwt_2d_radix8_forward_inplace / nwt_2d_radix8_backward_inplace
 * (thirdparty/phantom-fhe/include/ntt.cuh:47-99) as called by
 * moai::Evaluator::transform_to_ntt_inplace / transform_from_ntt_inplace
 * (src/include/source/ckks_evaluator_parallel.cuh:396-442). */
int shm_ntt_forward(const shm_context *ctx, uint64_t *data, uint32_t n_polys, uint32_t L, void *stream);
int shm_ntt_inverse(const shm_context *ctx, uint64_t *data, uint32_t n_polys, uint32_t L, void *stream);

/* out = a + b, a - b, -a over n_polys polynomials of L limbs.
 * Replaces add_inplace / sub_inplace / negate (thirdparty/phantom-fhe/src/evaluate.cu:114-348). */
int shm_add(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys,
            uint32_t L, void *stream);
int shm_sub(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys,
            uint32_t L, void *stream);
/* Sum of two batches of n_cts ciphertexts of different sizes (a_size >= b_size, e.g. an
 * unrelinearised product and an ordinary ciphertext): out[ct][p] = a[ct][p] + b[ct][p] for
 * p < b_size, a[ct][p] above.  Replaces add_inplace on ciphertexts of different sizes
 * (thirdparty/phantom-fhe/src/evaluate.cu:114-160). */
int shm_add_sizes(const shm_context *ctx, const uint64_t *a, uint32_t a_size, const uint64_t *b, uint32_t b_size,
                  uint64_t *out, uint32_t n_cts, uint32_t L, void *stream);
int shm_negate(const shm_context *ctx, const uint64_t *a, uint64_t *out, uint32_t n_polys, uint32_t L, void *stream);

/* out[c] = ct[c] * pt for n_polys polynomials and one plaintext [L][N].
 * Replaces multiply_plain_inplace / multiply_plain_ntt (evaluate.cu:1237-1266). */
int shm_multiply_plain(const shm_context *ctx, const uint64_t *ct, const uint64_t *pt, uint64_t *out,
                       uint32_t n_polys, uint32_t L, void *stream);

/* Size-3 tensor product of n_cts ciphertext pairs: out [n_cts][3][L][N].
 * Replaces bgv_ckks_multiply -> tensor_prod_2x2_rns_poly (evaluate.cu:350-402). */
int shm_multiply(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_cts,
                 uint32_t L, void *stream);

/* Sum of k size-3 tensor products: out[c] = sum_t A[t][c] x B[t][b_broadcast ? 0 : c] for n_cts
 * output ciphertexts [n_cts][3][L][N] (A[t]: [n_cts][2][L][N]; B[t]: one ciphertext when b_broadcast,
 * else [n_cts][2][L][N]); accumulate: add into out.  Equal to shm_multiply of every pair followed by
 * additions mod q.  Replaces the multiply + add_inplace loops of the attention's ct-ct products
 * (src/include/source/matrix_mul/Ct_ct_matrix_mul.cuh:10-120, :182-).  */
int shm_multiply_accumulate(const shm_context *ctx, const uint64_t *const *A, const uint64_t *const *B, uint32_t k,
                            int b_broadcast, uint64_t *out, uint32_t n_cts, uint32_t L, int accumulate, void *stream);

/* Rescale (floor division by the last prime) of n_polys polynomials, L -> L-1 limbs.
 * Replaces rescale_to_next / divide_and_round_q_last_ntt (evaluate.cu:1392-1443,
 * src/rns.cu:1157-1181). */
size_t shm_rescale_workspace_bytes(const shm_context *ctx, uint32_t n_polys, uint32_t L);
int shm_rescale(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
                void *workspace, size_t workspace_bytes, void *stream);

/* Rescale that allocates nothing: the same computation and result as
 * shm_rescale, for callers that cannot call cudaMalloc (hosts whose own pool
 * owns all device memory, latency-critical paths that cannot take cudaMalloc's
 * implicit synchronisation, FFI callers without a device allocator).  Scratch
 * comes from a fixed 32 MiB device array inside the library, which every GPU
 * that loads the library holds until exit; requests needing more than
 * shm_rescale_noalloc_max_words() words (n_polys * L * N) fail with SHM_EINVAL.
 * The first call on a device looks up the array's device address (make that
 * first call before any stream capture).  All calls share the one array, so
 * calls that overlap on the GPU (other streams, other threads) race; the array
 * needs no clearing (every call overwrites what it reads).
 * No counterpart in the reference: its rescale allocates per call. */
size_t shm_rescale_noalloc_max_words(void);
int shm_rescale_noalloc(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
                        void *stream);

/* Key switch of n_cts polynomials d [n_cts][L][N]: out (a [n_cts][2][L][N] buffer)
 * receives (cx0, cx1).  Replaces keyswitch_inplace's modup / inner product /
 * moddown (src/eval_key_switch.cu:91-178). */
size_t shm_keyswitch_workspace_bytes(const shm_context *ctx, uint32_t n_cts, uint32_t L);
int shm_keyswitch(const shm_context *ctx, const uint64_t *d, const uint64_t *key, uint64_t *out, uint32_t n_cts,
                  uint32_t L, void *workspace, size_t workspace_bytes, void *stream);

/* Relinearize n_cts size-3 ciphertexts [n_cts][3][L][N] into [n_cts][2][L][N].
 * Replaces relinearize_inplace (evaluate.cu:1358-1390). */
int shm_relinearize(const shm_context *ctx, const uint64_t *ct3, const uint64_t *relin_key, uint64_t *out,
                    uint32_t n_cts, uint32_t L, void *workspace, size_t workspace_bytes, void *stream);

/* Relinearize and rescale n_cts size-3 ciphertexts [n_cts][3][L][N] (2 <= L) into
 * [n_cts][2][L-1][N] with one ModDown by S = q_{L-1} P instead of a ModDown by P and a
 * rescale by q_{L-1}: out = floor((P c + <ModUp(c2), key>) / S), the conversion of the S
 * limbs made exact by its overflow count.  Equal to shm_relinearize + shm_rescale (the
 * reference's relinearize_inplace then rescale_to_next, evaluate.cu:1358-1443) except for
 * a coefficient whose sum lies within n_p + 1 of a multiple of q_{L-1} P (probability about
 * n_p / q_{L-1}; the result is then one less).  Saves the rescale's INTT and one forward NTT
 * of 2 (L - 1) limbs.  Workspace as shm_keyswitch_workspace_bytes(n_cts, L); out must not
 * overlap ct3. */
int shm_relinearize_rescale(const shm_context *ctx, const uint64_t *ct3, const uint64_t *relin_key, uint64_t *out,
                            uint32_t n_cts, uint32_t L, void *workspace, size_t workspace_bytes, void *stream);

/* Apply the automorphism X -> X^galois_elt with its key to n_cts ciphertexts.
 * Replaces apply_galois_inplace (evaluate.cu:1586-1647). */
int shm_apply_galois(const shm_context *ctx, const uint64_t *ct, uint32_t galois_elt, const uint64_t *galois_key,
                     uint64_t *out, uint32_t n_cts, uint32_t L, void *workspace, size_t workspace_bytes,
                     void *stream);
/* The automorphism X -> X^galois_elt of n_rows NTT-form polynomials of N words each, without key
 * switching (a permutation of the evaluation points; any prime per row): used on secrets to form
 * Galois keys on the device (generate_one_kswitch_key's s(X^elt), secretkey.cu:328-373, computed
 * there from the coefficients).  out must not overlap in. */
int shm_permute_galois(const shm_context *ctx, const uint64_t *in, uint32_t galois_elt, uint64_t *out,
                       uint32_t n_rows, void *stream);

/* Hoisted automorphisms of the same n_cts ciphertexts: ModUp of c1 once, then for
 * each of n_elts Galois elements the permuted inner product with keys[e] and
 * ModDown: outs[e] = (sigma(c0) + cx0, cx1).  keys / outs are host arrays of
 * device pointers; outputs must not alias the input.  Counterpart of the
 * reference's hoisted rotations (thirdparty/phantom-fhe/src/evaluate.cu:1727-1920),
 * used here for the baby steps of the bootstrapping linear transforms.  Decrypts
 * like shm_apply_galois; the limbs differ in the ModUp error term, so bit-exact
 * parity for this entry point is against the oracle's hoisted restatement. */
size_t shm_apply_galois_hoisted_workspace_bytes(const shm_context *ctx, uint32_t n_cts, uint32_t L);
int shm_apply_galois_hoisted(const shm_context *ctx, const uint64_t *ct, uint32_t n_elts, const uint32_t *elts,
                             const uint64_t *const *keys, uint64_t *const *outs, uint32_t n_cts, uint32_t L,
                             void *workspace, size_t workspace_bytes, void *stream);
/* Shared-a batches (multi-secret RLWE): n_groups groups of n_members ciphertexts,
 * each group stored as [n_members + 1][L][N] = (b_0 .. b_{n-1}, a) with
 * b_i + a s'_i ~ m_i (src/include/source/bootstrapping/SharedACiphertext.cuh:9-21).
 *
 * Sh-Rot of every group by each of n_elts Galois elements with one ModUp of the
 * shared a (hoisted): keys[e] is [dnum][n_members + 1][QP][N] (halves B_0..B_{n-1}, A),
 * outs[e] receives the rotated batch.  Replaces shared_a_rotate
 * (src/include/source/bootstrapping/ShRotate.cu:201-257). */
size_t shm_shared_rotate_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members, uint32_t L);
int shm_shared_rotate_hoisted(const shm_context *ctx, const uint64_t *sh, uint32_t n_groups, uint32_t n_members,
                              uint32_t n_elts, const uint32_t *elts, const uint64_t *const *keys, uint64_t *const *outs,
                              uint32_t L, void *workspace, size_t workspace_bytes, void *stream);
/* Sh-Rot of every group by one Galois element in the reference's order: the automorphism
 * on a and every b first, then one ModUp of the rotated a, the n + 1 inner products and
 * ModDowns (shared_a_rotate, ShRotate.cu:201-257; bit for bit the reference's limbs).  The
 * hoisted entry point above applies the automorphism to the extended digits after the
 * ModUp instead (one ModUp for every element): the same rotation up to the base
 * conversion's overflow multiples of Q, so it decrypts the same but its limbs differ. */
size_t shm_shared_rotate_one_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                             uint32_t L);
int shm_shared_rotate(const shm_context *ctx, const uint64_t *sh, uint32_t n_groups, uint32_t n_members, uint32_t elt,
                      const uint64_t *key, uint64_t *out, uint32_t L, void *workspace, size_t workspace_bytes,
                      void *stream);
/* FmtSwitch forward: n_groups * n_members ordinary ciphertexts [.][2][L][N] under s
 * -> shared-a batch [n_groups][n_members + 1][L][N] under s'_i, with the format key
 * [n_members][n_members + 1][QP][N] (halves B_fmt[j][0..n-1], a_fmt[j]); the a_j are
 * extended exactly from Ql to QlP.  Replaces fmt_switch_forward
 * (src/include/source/bootstrapping/FmtSwitch.cu:276-394). */
size_t shm_fmt_switch_forward_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                              uint32_t L);
int shm_fmt_switch_forward(const shm_context *ctx, const uint64_t *cts, uint32_t n_groups, uint32_t n_members,
                           const uint64_t *key, uint64_t *out, uint32_t L, void *workspace, size_t workspace_bytes,
                           void *stream);
/* FmtSwitch backward: shared-a batch -> n_groups * n_members ordinary ciphertexts
 * under s, keys[i] the switching key s'_i -> s ([dnum][2][QP][N]); one ModUp of each
 * shared a serves all members.  Replaces fmt_switch_backward (FmtSwitch.cu:396-429). */
size_t shm_fmt_switch_backward_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                               uint32_t L);
int shm_fmt_switch_backward(const shm_context *ctx, const uint64_t *sh, uint32_t n_groups, uint32_t n_members,
                            const uint64_t *const *keys, uint64_t *out, uint32_t L, void *workspace,
                            size_t workspace_bytes, void *stream);

/* ---- the extended basis QlP (double-hoisted linear transforms) ----
 * An extended polynomial at level L has L + n_p limbs: the Q limbs 0..L-1 under q_0..q_{L-1},
 * then the special primes p_0..p_{n_p-1}.  It stands for ModDown of itself, so the key
 * switches of a baby-step giant-step transform can stay in QlP and be brought down once
 * per transform (Bossuat et al.'s double hoisting); the reference ModDowns after every
 * rotation (ShRotate.cu:201-257, Bootstrapper.cu:2168-2340).
 * shm_extend: out = P * in (n_polys polynomials of L limbs -> L + n_p limbs, P limbs 0).
 * shm_add_ext: out = a + b over extended polynomials.
 * shm_moddown_ext: out [n_polys][L][N] = ModDown(ext); the P limbs of ext are overwritten.
 * shm_multiply_plain_accumulate_ext: as shm_multiply_plain_accumulate over extended X[t]
 *   and plaintexts P[t] of L + n_p limbs.
 * shm_lift_signed_ext / shm_ntt_forward_ext: signed coefficients -> extended residues / NTT
 *   of extended polynomials (plaintexts for the above).
 * shm_shared_rotate_ext: Sh-Rot of shared-a groups with extended outputs outs[e]
 *   [n_groups][n_members+1][L+n_p][N] (no ModDown); the input is ordinary groups
 *   [n_groups][n_members+1][L][N] (in_ext = 0) or extended groups (in_ext = 1, whose a rows
 *   are brought down once before the ModUp). */
int shm_extend(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
               void *stream);
int shm_add_ext(const shm_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys,
                uint32_t L, void *stream);
size_t shm_moddown_ext_workspace_bytes(const shm_context *ctx, uint32_t n_polys, uint32_t L);
int shm_moddown_ext(const shm_context *ctx, uint64_t *ext, uint64_t *out, uint32_t n_polys, uint32_t L,
                    void *workspace, size_t workspace_bytes, void *stream);
int shm_multiply_plain_accumulate_ext(const shm_context *ctx, const uint64_t *const *X, const uint64_t *const *P,
                                      uint32_t k, uint64_t *out, uint32_t n_polys, uint32_t L, int accumulate,
                                      void *stream);
int shm_lift_signed_ext(const shm_context *ctx, const int64_t *coeffs, uint64_t *out, uint32_t n_polys, uint32_t L,
                        void *stream);
int shm_ntt_forward_ext(const shm_context *ctx, uint64_t *data, uint32_t n_polys, uint32_t L, void *stream);
size_t shm_shared_rotate_ext_workspace_bytes(const shm_context *ctx, uint32_t n_groups, uint32_t n_members,
                                             uint32_t L);
int shm_shared_rotate_ext(const shm_context *ctx, const uint64_t *in, int in_ext, uint32_t n_groups,
                          uint32_t n_members, uint32_t n_elts, const uint32_t *elts, const uint64_t *const *keys,
                          uint64_t *const *outs, uint32_t L, void *workspace, size_t workspace_bytes, void *stream);
/* Galois element of a rotation by `step` slots (0 = conjugation).
 * Replaces PhantomGaloisTool::get_elt_from_step (src/galois.cu:47-91). */
uint32_t shm_galois_elt_from_step(const shm_context *ctx, int step);
/* HRotate: shm_apply_galois with shm_galois_elt_from_step(step).
 * Replaces moai::Evaluator::rotate_vector_inplace (ckks_evaluator_parallel.cuh:341-347). */
int shm_rotate(const shm_context *ctx, const uint64_t *ct, int step, const uint64_t *galois_key, uint64_t *out,
               uint32_t n_cts, uint32_t L, void *workspace, size_t workspace_bytes, void *stream);

/* out = a * s (per-limb scalar residues s[0..L), host array) over n_polys polynomials.
 * Replaces multiply_const_inplace's constant multiply (ckks_evaluator_parallel.cuh:245-262;
 * a constant plaintext in NTT form is one residue per limb). */
int shm_multiply_scalar(const shm_context *ctx, const uint64_t *a, const uint64_t *scalars, uint64_t *out,
                        uint32_t n_polys, uint32_t L, void *stream);
/* c0 of each of n_cts ciphertexts gets + s[limb]; c1 is copied.
 * Replaces add_const_inplace (ckks_evaluator_parallel.cuh:263-280). */
int shm_add_scalar(const shm_context *ctx, const uint64_t *a, const uint64_t *scalars, uint64_t *out,
                   uint32_t n_cts, uint32_t L, void *stream);
/* out (+)= sum_t X[t] * P[t] over k terms: X[t] are [n_polys][L][N] device
 * buffers, P[t] are [L][N] plaintexts (host arrays of device pointers).
 * Replaces the per-diagonal multiply_plain + add_inplace inner loop of
 * Bootstrapper::bsgs_linear_transform (src/include/source/bootstrapping/Bootstrapper.cu:2168-2340). */
int shm_multiply_plain_accumulate(const shm_context *ctx, const uint64_t *const *X, const uint64_t *const *P,
                                  uint32_t k, uint64_t *out, uint32_t n_polys, uint32_t L, int accumulate,
                                  void *stream);
/* out = sum_t w[t] * X[t] + w0 for n_cts size-2 ciphertexts at L limbs, one pass: X[t] is
 * [n_cts][2][X_levels[t]][N] with X_levels[t] >= L (only its first L limbs are read, so no
 * limb drop is needed), w is [k][L] residues (the weight of term t mod each prime), w0 is [L]
 * residues added to c0 (NULL: none); k <= 8, L <= 64.  Replaces the mod_switch_to +
 * multiply_const + add_inplace per term and the final add_const of a polynomial leaf
 * (src/include/source/ckks_evaluator_parallel.cuh:245-280, thirdparty/phantom-fhe/src/
 * evaluate.cu:114-160); the sums mod q are the same, so the result is identical. */
int shm_linear_combination(const shm_context *ctx, const uint64_t *const *X, const uint32_t *X_levels,
                           const uint64_t *w, uint32_t k, const uint64_t *w0, uint64_t *out, uint32_t n_cts,
                           uint32_t L, void *stream);
/* Mod-raise n_polys one-limb polynomials (mod q0, NTT form) to L limbs by the
 * centred lift.  Replaces Bootstrapper::modraise_inplace (Bootstrapper.cu:3271-3356). */
size_t shm_modraise_workspace_bytes(const shm_context *ctx, uint32_t n_polys);
int shm_modraise(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
                 void *workspace, size_t workspace_bytes, void *stream);
/* Keep the first L_out of L_in limbs of n_polys polynomials (modulus drop without
 * rescale).  Replaces mod_switch_drop_to_next / mod_switch_to_inplace (evaluate.cu:1445-1520). */
int shm_drop_limbs(const shm_context *ctx, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L_in,
                   uint32_t L_out, void *stream);

/* Rotation-free ct-pt matmul: Y[o] = sum_i X[i] * W[i][o] over n_in input
 * ciphertexts X [n_in][2][L][N] and signed integer weights W [n_in][n_out]
 * (the encoded constants round(w * scale)); Y is [n_out][2][L][N] before the
 * rescale.  Replaces the multiply_plain + add_inplace loop of
 * ct_pt_matrix_mul_wo_pre (src/include/source/matrix_mul/Ct_pt_matrix_mul.cuh:112-158). */
size_t shm_ctpt_matmul_workspace_bytes(const shm_context *ctx, uint32_t n_in, uint32_t n_out, uint32_t L);
/* Computed on the INT8 tensor cores (tcgen05.mma kind::i8) through a small-modulus
 * residue system: exact for |W| < 2^40 (larger weights: SHM_EINVAL).  The call
 * reads W back to the host once to size the residue system, so it synchronises
 * `stream`. */
int shm_ctpt_matmul(const shm_context *ctx, const uint64_t *X, const int64_t *W, uint64_t *Y, uint32_t n_in,
                    uint32_t n_out, uint32_t L, void *workspace, size_t workspace_bytes, void *stream);
/* The same contraction on the CUDA cores (64-bit multiply-accumulate, |W| < 2^40):
 * the plain path the tensor-core kernel is measured against. */
int shm_ctpt_matmul_cuda_core(const shm_context *ctx, const uint64_t *X, const int64_t *W, uint64_t *Y,
                              uint32_t n_in, uint32_t n_out, uint32_t L, void *stream);

/* ---- device memory (the allocator of the host library, include/shmoai/host.hpp) ----
 * Stream-ordered blocks from a per-context pool that keeps freed blocks for reuse, so
 * the pipeline's many short-lived buffers cost no driver calls or synchronisation.
 * Replaces the reference's cuda_auto_ptr over its cudaMallocAsync pool
 * (thirdparty/phantom-fhe/include/cuda_wrapper.cuh:78-211). */
#define SHM_COPY_H2D 0
#define SHM_COPY_D2H 1
#define SHM_COPY_D2D 2
int shm_malloc(const shm_context *ctx, size_t bytes, void **out, void *stream);
int shm_free(const shm_context *ctx, void *ptr, void *stream);
/* Copies involving host memory return when the copy is done; device-to-device copies are
 * asynchronous on `stream`. */
int shm_memcpy(const shm_context *ctx, void *dst, const void *src, size_t bytes, int kind, void *stream);
int shm_synchronize(const shm_context *ctx, void *stream);
/* Bytes the context's pool holds from the driver, bytes in use, and the high-water mark of
 * bytes in use (reset to the current use when reset_high != 0); any pointer may be NULL. */
int shm_pool_usage(const shm_context *ctx, size_t *reserved, size_t *used, size_t *used_high, int reset_high);
/* A non-blocking stream on the context's device (the serving loop runs one per slot). */
int shm_stream_create(const shm_context *ctx, void **stream);
int shm_stream_destroy(const shm_context *ctx, void *stream);

/* ---- CUDA graphs of whole operation sequences ----
 * No reference counterpart: the reference issues every kernel from the host per call
 * (thirdparty/phantom-fhe/src/evaluate.cu).  Between shm_graph_begin and shm_graph_end the
 * calls that work on `stream` are recorded instead of run; shm_graph_launch then replays all
 * of them with one launch, on any stream.  The recorded calls must make no host round trip
 * (no host copies, no synchronisation) and must free on the stream, before shm_graph_end,
 * every buffer they allocate with shm_malloc; run the sequence once outside the capture first
 * so that lazily built tables exist.  `stream` must come from shm_stream_create (the legacy
 * default stream cannot be captured).  shm_graph_begin releases the context pool's unused
 * blocks: the graph's own allocations come from the device's graph memory. */
typedef struct shm_graph shm_graph;
int shm_graph_begin(const shm_context *ctx, void *stream);
int shm_graph_end(const shm_context *ctx, void *stream, shm_graph **out);
int shm_graph_launch(const shm_graph *g, void *stream);
/* kernels recorded in the graph (added to shm_kernel_launches by every replay) */
uint64_t shm_graph_kernels(const shm_graph *g);
void shm_graph_destroy(shm_graph *g);

/* ---- autotuning of kernel tiles ----
 * No reference counterpart (its launch shapes are fixed).  Times every candidate of one
 * knob with CUDA events on scratch data shaped like the caller's workload and keeps the
 * fastest for this context; later calls on any stream use it.  Synchronises the device.
 *   SHM_TUNE_NTT_TILE  tile variant of the NTT kernels, candidates 0..3 = (columns per CTA,
 *                      minimum resident CTAs per SM) (16, 4), (16, 3), (8, 8), (8, 6);
 *                      workload: forward + inverse NTT of `size` limbs.
 *   SHM_TUNE_IP_CHUNK  shared memory of one Sh-Rot inner-product block, candidates 0..3 =
 *                      16, 32, 64, 96 KB (more groups of a chunk share each key read);
 *                      workload: `size` groups of `members` at `level` primes.
 * times (NULL or room for `cap` values) receives the candidates' milliseconds in order;
 * *chosen the winner's index. */
#define SHM_TUNE_NTT_TILE 0
#define SHM_TUNE_IP_CHUNK 1
int shm_autotune(shm_context *ctx, int knob, uint32_t size, uint32_t level, uint32_t members, float *times,
                 uint32_t cap, uint32_t *chosen);
/* the candidate index a knob uses now / force one (e.g. a stored tuning result) */
int shm_tune_get(const shm_context *ctx, int knob, uint32_t *index);
int shm_tune_set(shm_context *ctx, int knob, uint32_t index);

/* ---- sampling (key generation, encryption) ----
 * Counter-based: value i of a call is a function of (seed, i) only, so the GPU and the
 * CPU restatement draw identical keys and ciphertexts.  Distributions as in the
 * reference's samplers (thirdparty/phantom-fhe/src/prng.cu:142-240); the streams differ.
 * Uniform residues: out [n_polys][L][N], limb i uniform mod prime i (L <= nq + np). */
int shm_sample_uniform(const shm_context *ctx, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t seed,
                       void *stream);
/* Centred binomial over 21 + 21 bits (sigma ~ 3.24), one integer polynomial per poly,
 * written as residues mod each of the first L primes (coefficient form). */
int shm_sample_cbd(const shm_context *ctx, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t seed,
                   void *stream);
/* ---- canonical-embedding encode / decode (FP64 on the GPU; the library's only
 * floating-point work).  Replaces PhantomCKKSEncoder::encode_internal / decode_internal
 * (thirdparty/phantom-fhe/src/ckks.cu:89-246, special FFT fft.cu:358-439) for a batch of
 * vectors in one call.  Device arrays: re, im [n_vectors][n_values] slot values
 * (n_values <= N/2, the rest zero) -> coeffs [n_vectors][N] = round-half-even of the
 * coefficients of the polynomial whose slots are z * scale; SHM_EINVAL when one reaches 2^62
 * (the call then synchronises the stream).  decode: coeffs [n_vectors][N] (real, centred)
 * -> re, im [n_vectors][N/2] slot values / scale.  The FFT is the host encoder's
 * (shmoai::Encoder::encode_float / decode) operation for operation, so both give the same
 * bits. */
size_t shm_encode_workspace_bytes(const shm_context *ctx, uint32_t n_vectors);
int shm_encode(const shm_context *ctx, const double *re, const double *im, uint32_t n_vectors, uint32_t n_values,
               double scale, int64_t *coeffs, void *workspace, size_t workspace_bytes, void *stream);
int shm_decode(const shm_context *ctx, const double *coeffs, uint32_t n_vectors, double scale, double *re, double *im,
               void *workspace, size_t workspace_bytes, void *stream);
/* Signed coefficients [n_polys][N] (device) -> residues [n_polys][L][N] (coefficient form).
 * Replaces the signed decomposition of the encoder (rns_base.cu:51-200). */
int shm_lift_signed(const shm_context *ctx, const int64_t *coeffs, uint64_t *out, uint32_t n_polys, uint32_t L,
                    void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SHMOAI_CKKS_H */
