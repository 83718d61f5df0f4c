// Hybrid (dnum-digit) key switching for a batch of polynomials sharing one key.
//
// Reference semantics (bit-identical): thirdparty/phantom-fhe/src/eval_key_switch.cu:91-178
//   ModUp     src/rns_bconv.cu:530-628: per digit b (limbs [b*alpha, min((b+1)*alpha, L))),
//             y_i = INTT(d_i) * qhat_i^-1 mod q_i; every other limb t_j of QlP gets
//             sum_i y_i * (qhat_i mod t_j) mod t_j (no correction term), then NTT;
//             the digit's own limbs keep d_i unchanged.
//   product   src/eval_key_switch.cu:12-66: cx_h[j] = sum_b up_b[j] * key_b[h][prime(j)].
//   ModDown   src/rns_bconv.cu:776-828: z_k = INTT(cx_h[L+k]) * phat_k^-1,
//             delta_j = NTT(sum_k z_k * (phat_k mod q_j)), out = (cx_h[j] - delta_j) * P^-1.
//
// Batch layout: the key is read once per coefficient for all n_cts polynomials
// (the inner-product kernel loops over the batch with the key digits in registers).
#include "core.hpp"

namespace shm {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxAlpha = 16;
constexpr int kMaxBeta = 16;

// acc[ct][h][j][k] = sum_b up[ct][b][j][perm[k]] * key[b][h][prime(j)][k]   (perm = identity if null)
// An NTT-domain automorphism maps every aligned block of 32 slots onto an aligned block
// of 32 slots, so the permuted read of a warp stays within one 256-byte segment.
// B = beta at compile time: the key rows held in registers for the whole batch are
// exactly 2B words, so small digit counts keep more warps resident.
template <int B, bool S52>
__global__ void inner_product_kernel(const uint64_t *__restrict__ up, const uint64_t *__restrict__ key,
                                     uint64_t *__restrict__ acc, uint32_t n_cts, uint32_t L, uint32_t np, uint32_t nq,
                                     uint32_t log_n, const PrimeConst *__restrict__ pc,
                                     const uint32_t *__restrict__ perm) {
    const uint32_t j = blockIdx.y;
    const uint32_t k = blockIdx.x * kThreads + threadIdx.x;
    const uint32_t ks = perm ? __ldg(perm + k) : k;
    const size_t n = (size_t)1 << log_n;
    const uint32_t LP = L + np, QP = nq + np;
    const uint32_t pj = j < L ? j : nq + (j - L);
    const PrimeConst p = pc[pj];
    uint64_t k0[B], k1[B];
#pragma unroll
    for (int b = 0; b < B; b++) {
        const uint64_t *kb = key + (size_t)b * 2 * QP * n;
        k0[b] = kb[(size_t)pj * n + k];
        k1[b] = kb[((size_t)QP + pj) * n + k];
    }
    for (uint32_t ct = 0; ct < n_cts; ct++) {
        const uint64_t *u = up + (size_t)ct * B * LP * n + (size_t)j * n + ks;
        uint64_t v[B];
#pragma unroll
        for (int b = 0; b < B; b++) v[b] = u[(size_t)b * LP * n];
        Acc<S52> a0, a1;
#pragma unroll
        for (int b = 0; b < B; b++) {
            a0.add(v[b], k0[b]);
            a1.add(v[b], k1[b]);
        }
        uint64_t *o = acc + (size_t)ct * 2 * LP * n + (size_t)j * n + k;  // output in natural slot order
        o[0] = barrett(a0.get(), p);
        o[(size_t)LP * n] = barrett(a1.get(), p);
    }
}

template <bool S52>
void launch_inner_product(dim3 grid, cudaStream_t st, const uint64_t *up, const uint64_t *key, uint64_t *acc,
                          uint32_t n_cts, uint32_t L, uint32_t np, uint32_t nq, uint32_t beta, uint32_t log_n,
                          const PrimeConst *pc, const uint32_t *perm) {
#define SHM_IP_CASE(B)                                                                                               \
    case B:                                                                                                          \
        inner_product_kernel<B, S52><<<grid, kThreads, 0, st>>>(up, key, acc, n_cts, L, np, nq, log_n, pc, perm); \
        break;
    switch (beta) {
        SHM_IP_CASE(1) SHM_IP_CASE(2) SHM_IP_CASE(3) SHM_IP_CASE(4) SHM_IP_CASE(5) SHM_IP_CASE(6) SHM_IP_CASE(7)
        SHM_IP_CASE(8) SHM_IP_CASE(9) SHM_IP_CASE(10) SHM_IP_CASE(11) SHM_IP_CASE(12) SHM_IP_CASE(13)
        SHM_IP_CASE(14) SHM_IP_CASE(15) SHM_IP_CASE(16)
        default:
            throw std::invalid_argument("key-switching digit count out of range");
    }
#undef SHM_IP_CASE
}

// the inner product for one context: Acc<true> when every prime is below 2^52
void launch_ip(const Context &c, uint32_t n_cts, uint32_t L, const uint64_t *up, const uint64_t *key, uint64_t *acc,
               const uint32_t *perm, cudaStream_t st) {
    const uint32_t np = c.np, beta = (L + np - 1) / np, LP = L + np;
    const dim3 grid(c.n / kThreads, LP);
    SHM_LAUNCHED(1);
    if (c.s52)
        launch_inner_product<true>(grid, st, up, key, acc, n_cts, L, np, c.nq, beta, c.log_n, c.pc, perm);
    else
        launch_inner_product<false>(grid, st, up, key, acc, n_cts, L, np, c.nq, beta, c.log_n, c.pc, perm);
    SHM_CUDA(cudaGetLastError());
}

// the fused ModDown's addressing for a KsOutput (out1 = out0 + L N, add1 = add0 + L N or null,
// one stride for out and add; add0 read through add0_perm when set)
ModDownIO moddown_io(const Context &c, const uint64_t *acc, const KsOutput &o) {
    ModDownIO md;
    md.acc = acc;
    md.conv = c.moddown_conv;
    md.pinv = c.p_inv;
    md.out = o.out0;
    md.out_ct = (long long)o.stride;
    md.out_h = (long long)(o.out1 - o.out0);
    md.add = o.add0;
    md.add_ct = (long long)o.stride;
    md.add_h = o.add1 ? (long long)(o.add1 - o.add0) : 0;
    md.n_add = o.add0 ? (o.add1 ? 2 : 1) : 0;
    md.perm = o.add0_perm;
    md.n_perm = 1;
    md.H = 2;
    md.np = c.np;
    md.s52 = c.s52 ? 1 : 0;
    return md;
}


// acc[ct][h][row] += (P mod q) * ct3[ct][h][row] for h = 0, 1: the q_{L-1} limb of P c added
// before that limb joins the special primes of the ModDown by q_{L-1} P
__global__ void add_p_times_kernel(uint64_t *__restrict__ acc, const uint64_t *__restrict__ ct3, uint32_t L,
                                   uint32_t LP, uint32_t row, uint64_t pm, uint64_t pms, uint64_t q, uint32_t log_n) {
    const uint32_t k = blockIdx.x * kThreads + threadIdx.x, poly = blockIdx.y, ct = poly >> 1, h = poly & 1;
    uint64_t *a = acc + (((size_t)poly * LP + row) << log_n) + k;
    const uint64_t x = ct3[(((size_t)ct * 3 + h) * L + row << log_n) + k];
    *a = add_mod(*a, shoup(x, pm, pms, q), q);
}

// v = floor(sum_k z_k / s_k) for the INTT'd limbs z_k of S (rows first .. first + ns - 1 of
// each [LP][N] polynomial, z_k = [y (S/s_k)^-1]_{s_k}): sum_k z_k (S / s_k) = [y]_S + v S, so
// subtracting v S makes the conversion exact.  The sum is formed in double precision, one
// unfused multiply and add per term in k order (the oracle does the same); its error is
// below 2^-49, so v is wrong only when [y]_S / S lies that close to 0 or 1.
__global__ void overflow_count_kernel(const uint64_t *__restrict__ acc, uint8_t *__restrict__ v, uint32_t LP,
                                      uint32_t first, uint32_t ns, const double *__restrict__ inv_s, uint32_t log_n) {
    const uint32_t k = blockIdx.x * kThreads + threadIdx.x, poly = blockIdx.y;
    const uint64_t *z = acc + (((size_t)poly * LP + first) << log_n) + k;
    double f = 0.0;
    for (uint32_t i = 0; i < ns; i++) f = __dadd_rn(f, __dmul_rn(__ull2double_rn(z[(size_t)i << log_n]), __ldg(inv_s + i)));
    v[((size_t)poly << log_n) + k] = (uint8_t)f;
}

}  // namespace

void relin_rescale(const Context &c, const uint64_t *ct3, uint32_t n_cts, uint32_t L, const uint64_t *key,
                   uint64_t *out, uint64_t *ws, cudaStream_t st) {
    if (n_cts == 0) return;
    if (c.np == 0) throw std::invalid_argument("context has no special primes: key switching unavailable");
    if (L < 2 || L > c.nq) throw std::invalid_argument("relinearize-rescale needs 2 <= L <= n_q");
    const uint32_t np = c.np, beta = (L + np - 1) / np, LP = L + np;
    if (beta > c.dnum) throw std::invalid_argument("level needs more key digits than the key holds");
    if (np > kMaxAlpha || beta > kMaxBeta || LP > 64) throw std::invalid_argument("key-switching shape too large");
    const size_t n = c.n, ln = (size_t)L * n;
    uint64_t *x = ws;
    uint64_t *up = x + (size_t)n_cts * L * n;
    uint64_t *acc = up + (size_t)n_cts * beta * LP * n;
    uint64_t *delta = up;
    const LevelKS &ks = c.ks[L];

    modup_into(c, ct3 + 2 * ln, 3 * ln, n_cts, L, x, up, st);
    launch_ip(c, n_cts, L, up, key, acc, nullptr, st);
    // y = P c + ks over QlP: P c vanishes mod every p_k; on the limbs j < L - 1 it is folded
    // into the ModDown's store as c_j q_{L-1}^-1 (= P c_j S^-1); limb L - 1 gets it here
    const uint64_t ql = c.primes[L - 1];
    SHM_LAUNCHED(1);
    add_p_times_kernel<<<dim3(c.n / kThreads, n_cts * 2), kThreads, 0, st>>>(
        acc, ct3, L, LP, L - 1, c.h_p_mod[2 * (L - 1)], c.h_p_mod[2 * (L - 1) + 1], ql, c.log_n);
    SHM_CUDA(cudaGetLastError());
    // ModDown by S = q_{L-1} P: INTT of rows L-1 .. LP-1 scaled by (S / s_k)^-1, the overflow
    // count of the conversion, exact conversion to the L - 1 remaining primes, NTT,
    // (y_j - conv_j) S^-1 = floor(y / S)
    LimbMap mp;
    for (uint32_t r = 0; r < 512; r++)
        mp.prime[r] = r == L - 1 ? (uint8_t)(L - 1) : (r >= L && r < LP) ? (uint8_t)(c.nq + (r - L)) : 255;
    ntt_inverse(c, acc, n_cts * 2 * LP, LP, mp, ks.rr_scale, st, L - 1);
    uint8_t *vrow = reinterpret_cast<uint8_t *>(x);  // x is free after the ModUp: [n_cts][2][N] bytes
    SHM_LAUNCHED(1);
    overflow_count_kernel<<<dim3(c.n / kThreads, n_cts * 2), kThreads, 0, st>>>(acc, vrow, LP, L - 1, np + 1,
                                                                                ks.rr_inv_s, c.log_n);
    SHM_CUDA(cudaGetLastError());
    ModDownIO md;
    md.acc = acc;
    md.conv = ks.rr_conv;
    md.pinv = ks.rr_sinv;
    md.out = out;
    md.out_ct = (long long)(2 * (L - 1) * n);
    md.out_h = (long long)((L - 1) * n);
    md.add = ct3;
    md.add_ct = (long long)(3 * ln);
    md.add_h = (long long)ln;
    md.add_mul = c.rescale_inv + (size_t)(L - 1) * c.nq * 2;
    md.n_add = 2;
    md.H = 2;
    md.np = np + 1;
    md.s52 = c.s52 ? 1 : 0;
    md.vrow = vrow;
    md.vs = ks.rr_vs;
    ntt_forward_moddown(c, md, delta, n_cts * 2, L - 1, st);
}

size_t keyswitch_ws_words(const Context &c, uint32_t n_cts, uint32_t L) {
    const uint32_t beta = (L + c.np - 1) / c.np, LP = L + c.np;
    return (size_t)n_cts * c.n * (L + (size_t)beta * LP + 2 * (size_t)LP);
}

void keyswitch(const Context &c, const uint64_t *d, size_t d_stride, uint32_t n_cts, uint32_t L, const uint64_t *key,
               const KsOutput &o, uint64_t *ws, cudaStream_t st) {
    if (n_cts == 0) return;
    if (c.np == 0) throw std::invalid_argument("context has no special primes: key switching unavailable");
    if (L < 1 || L > c.nq) throw std::invalid_argument("level out of range");
    const uint32_t np = c.np, beta = (L + np - 1) / np, LP = L + np;
    if (beta > c.dnum) throw std::invalid_argument("level needs more key digits than the key holds");
    if (np > kMaxAlpha || beta > kMaxBeta || LP > 64) throw std::invalid_argument("key-switching shape too large");
    const size_t n = c.n;
    uint64_t *x = ws;                                   // [n_cts][L][N]
    uint64_t *up = x + (size_t)n_cts * L * n;           // [n_cts][beta][LP][N]
    uint64_t *acc = up + (size_t)n_cts * beta * LP * n; // [n_cts][2][LP][N]
    uint64_t *delta = up;                               // reuses up: [n_cts][2][L][N]

    // 1-3. ModUp: coefficient form scaled by qhat_i^-1, base conversion of each digit to
    // the rest of QlP, NTT of the converted limbs (digit rows are already NTT form)
    modup_into(c, d, d_stride, n_cts, L, x, up, st);
    // 4. inner product with the key digits
    launch_ip(c, n_cts, L, up, key, acc, nullptr, st);
    // 5. ModDown: INTT of the P limbs (scaled by phat_k^-1), convert to Ql, NTT, combine
    LimbMap mp;
    for (uint32_t s = 0; s < 512; s++) mp.prime[s] = (s >= L && s < LP) ? (uint8_t)(c.nq + (s - L)) : 255;
    ntt_inverse(c, acc, n_cts * 2 * LP, LP, mp, c.moddown_scale, st, L);
    ntt_forward_moddown(c, moddown_io(c, acc, o), delta, n_cts * 2, L, st);
}

// ModUp of n_cts polynomials d (stride d_stride words) into up [n_cts][beta][LP][N]; x is
// an [n_cts][L][N] scratch.  Shared by the shared-a operations (shared.cu).
void modup_into(const Context &c, const uint64_t *d, size_t d_stride, uint32_t n_cts, uint32_t L, uint64_t *x,
                uint64_t *up, cudaStream_t st) {
    const uint32_t np = c.np, beta = (L + np - 1) / np, LP = L + np;
    if (np > kMaxAlpha || beta > kMaxBeta || LP > 64) throw std::invalid_argument("key-switching shape too large");
    const size_t n = c.n, ln = (size_t)L * n;
    const LevelKS &ks = c.ks[L];
    SHM_CUDA(cudaMemcpy2DAsync(x, ln * 8, d, d_stride * 8, ln * 8, n_cts, cudaMemcpyDeviceToDevice, st));
    ntt_inverse(c, x, n_cts * L, L, q_map(L), ks.modup_scale, st);
    LimbMap m;
    for (uint32_t s = 0; s < 512; s++) {
        if (s >= beta * LP) {
            m.prime[s] = 255;
            continue;
        }
        uint32_t b = s / LP, j = s % LP;
        bool own = j >= b * np && j < std::min((b + 1) * np, L);
        m.prime[s] = own ? 255 : (uint8_t)(j < L ? j : c.nq + (j - L));
    }
    // the conversion is computed in the forward NTT's load and the digits' own rows are copied by
    // the same launch: the converted limbs never go through HBM in coefficient form
    ModUpIO mu;
    mu.x = x;
    mu.d = d;
    mu.d_stride = (long long)d_stride;
    mu.conv = ks.modup_conv;
    mu.L = L;
    mu.np = np;
    mu.LP = LP;
    mu.s52 = c.s52 ? 1 : 0;
    ntt_forward_modup(c, mu, up, n_cts, beta, m, st);
}

size_t hoisted_ws_words(const Context &c, uint32_t n_cts, uint32_t L) {
    // x, up (kept for every element), acc and a separate delta
    return keyswitch_ws_words(c, n_cts, L) + (size_t)n_cts * 2 * L * c.n;
}

void apply_galois_hoisted(const Context &c, const uint64_t *ct, uint32_t n_cts, uint32_t L, uint32_t n_elts,
                          const uint32_t *elts, const uint64_t *const *keys, uint64_t *const *outs, uint64_t *ws,
                          cudaStream_t st) {
    if (n_cts == 0 || n_elts == 0) return;
    if (c.np == 0) throw std::invalid_argument("context has no special primes: key switching unavailable");
    if (L < 1 || L > c.nq) throw std::invalid_argument("level out of range");
    const uint32_t np = c.np, beta = (L + np - 1) / np, LP = L + np;
    if (beta > c.dnum) throw std::invalid_argument("level needs more key digits than the key holds");
    if (np > kMaxAlpha || beta > kMaxBeta || LP > 64) throw std::invalid_argument("key-switching shape too large");
    const size_t n = c.n, ln = (size_t)L * n;
    uint64_t *x = ws;
    uint64_t *up = x + (size_t)n_cts * L * n;
    uint64_t *acc = up + (size_t)n_cts * beta * LP * n;
    uint64_t *delta = acc + (size_t)n_cts * 2 * LP * n;  // up must survive every element
    const uint64_t *d = ct + ln;  // c1 of every ciphertext, stride 2 ln

    // ModUp once (identical to keyswitch steps 1-3)
    modup_into(c, d, 2 * ln, n_cts, L, x, up, st);
    LimbMap mp;
    for (uint32_t s = 0; s < 512; s++) mp.prime[s] = (s >= L && s < LP) ? (uint8_t)(c.nq + (s - L)) : 255;

    // per element: permuted inner product, ModDown, combine with sigma(c0)
    for (uint32_t e = 0; e < n_elts; e++) {
        const uint32_t *perm = const_cast<Context &>(c).perm(elts[e]);
        launch_ip(c, n_cts, L, up, keys[e], acc, perm, st);
        ntt_inverse(c, acc, n_cts * 2 * LP, LP, mp, c.moddown_scale, st, L);
        KsOutput o{outs[e], outs[e] + ln, ct, nullptr, 2 * ln, perm};
        ntt_forward_moddown(c, moddown_io(c, acc, o), delta, n_cts * 2, L, st);
    }
}

}  // namespace shm
