// Shared-a (multi-secret RLWE) batches: Sh-Rot, FmtSwitch forward and backward.
//
// A group of n ciphertexts is held as n + 1 polynomials [b_0 .. b_{n-1}, a] with
// b_i + a s'_i ~ m_i under auxiliary secrets s'_i (reference:
// src/include/source/bootstrapping/SharedACiphertext.cuh:9-21).  All three
// operations are "one ModUp-like extension of a shared polynomial, then H inner
// products against key halves, H ModDowns and a combine":
//
//   Sh-Rot (ShRotate.cu:201-257): extension = ModUp(a); key [dnum][n+1][QP][N] with
//     halves B_{g,0..n-1}, A_g; out b_i = sigma(b_i) + ModDown(<up, B_i>),
//     out a = ModDown(<up, A>).  Several rotation steps of the same batch share
//     one ModUp (hoisting; the automorphism is applied to the extended digits).
//   FmtSwitch forward (FmtSwitch.cu:276-394): the "digits" are the n members' a_j,
//     each extended exactly from Ql to QlP (floor-corrected CRT, FmtSwitch.cu:82-108);
//     key [n][n+1][QP][N] with halves B_fmt[j][0..n-1], a_fmt[j];
//     out b'_i = b_i + ModDown(<a_ext, B_fmt[:, i]>), a' = ModDown(<a_ext, a_fmt>).
//   FmtSwitch backward (FmtSwitch.cu:396-429): n ordinary key switches of the
//     shared a from s'_i to s, hoisted: one ModUp(a), per member one inner product
//     with its key [dnum][2][QP][N], ModDown, combine with b_i.
#include <mutex>

#include "core.hpp"
#include "host_math.hpp"

namespace shm {

namespace {

constexpr int kT = 256;
constexpr int kMaxB = 16;

// acc[ct][h][j][k] = sum_b up[ct][b][j][perm(k)] * key[b][h][prime(j)][k], h < H.
// A block handles `chunk` groups: each thread stages its own extended-digit words of those
// groups in shared memory (a column per thread, so no synchronisation), then, half by
// half, holds the key digits in registers and serves every group of the chunk: the key
// (n + 1 halves of dnum x QP limbs, far larger than L2 at the top level) is read once per
// chunk instead of once per group.
constexpr int kIpT = 128;
constexpr size_t kIpSmemMax = 96 * 1024;  // largest chunk the autotuner may pick

template <bool S52>
__global__ void __launch_bounds__(kIpT) ip_multi_kernel(const uint64_t *__restrict__ up,
                                                        const uint64_t *__restrict__ key, uint64_t *__restrict__ acc,
                                                        uint32_t n_cts, uint32_t chunk, uint32_t L, uint32_t np,
                                                        uint32_t nq, uint32_t beta, uint32_t H, uint32_t log_n,
                                                        const PrimeConst *__restrict__ pc,
                                                        const uint32_t *__restrict__ perm) {
    extern __shared__ uint64_t su[];  // [chunk * beta][kIpT]
    const uint32_t j = blockIdx.y;
    const uint32_t k = blockIdx.x * kIpT + threadIdx.x;
    const uint32_t ks = perm ? __ldg(perm + k) : k;
    const size_t n = (size_t)1 << log_n;
    const uint32_t LP = L + np, QP = nq + np;
    const uint32_t pj = j < L ? j : nq + (j - L);
    const PrimeConst p = pc[pj];
    const uint32_t c0 = blockIdx.z * chunk, nc = min(chunk, n_cts - c0);
    for (uint32_t ct = 0; ct < nc; ct++) {
        const uint64_t *up_c = up + (size_t)(c0 + ct) * beta * LP * n + (size_t)j * n + ks;
        for (uint32_t b = 0; b < beta; b++) su[(ct * beta + b) * kIpT + threadIdx.x] = up_c[(size_t)b * LP * n];
    }
    for (uint32_t h = 0; h < H; h++) {
        uint64_t kk[kMaxB];
        const uint64_t *kp = key + ((size_t)h * QP + pj) * n + k;
#pragma unroll
        for (int b = 0; b < kMaxB; b++)
            if (b < (int)beta) kk[b] = __ldg(kp + (size_t)b * H * QP * n);
        for (uint32_t ct = 0; ct < nc; ct++) {
            Acc<S52> a;
            const uint64_t *s = su + ct * beta * kIpT + threadIdx.x;
#pragma unroll
            for (int b = 0; b < kMaxB; b++)
                if (b < (int)beta) a.add(s[b * kIpT], kk[b]);
            acc[(((size_t)(c0 + ct) * H + h) * LP + j) * n + k] = barrett(a.get(), p);
        }
    }
}

struct Target {
    const uint64_t *key;  // [beta][H][QP][N]
    const uint32_t *perm;
    uint64_t *out;
    size_t out_ct, out_h;
    const uint64_t *add;
    size_t add_ct, add_h;
    uint32_t n_add;
};

// exact Ql -> P extension (floor-corrected CRT): x = sum_i y_i qhat_i - v Q, v = floor(sum_i y_i / q_i),
// y_i = [x_i qhat_i^-1]_{q_i} already in the coefficient buffer; writes the P rows of ext.
// v follows FmtSwitch.cu:86-106 operation for operation: the double sum of the correctly rounded
// quotients y_i / q_i in limb order (no contraction), truncated, plus one where the sum lies
// within 1e-9 below the next integer.
__global__ void exact_ext_kernel(const uint64_t *__restrict__ y, uint64_t *__restrict__ ext, const uint64_t *__restrict__ tab,
                                 const double *__restrict__ qd, uint32_t L, uint32_t np, uint32_t nq, uint32_t log_n,
                                 const PrimeConst *__restrict__ pc) {
    const uint32_t poly = blockIdx.y;
    const uint32_t k = blockIdx.x * kT + threadIdx.x;
    const size_t n = (size_t)1 << log_n;
    const uint64_t *yp = y + (size_t)poly * L * n + k;
    uint64_t yv[64];
    double frac = 0.0;
    for (uint32_t i = 0; i < L; i++) {
        yv[i] = yp[(size_t)i * n];
        frac = __dadd_rn(frac, __ddiv_rn((double)yv[i], qd[i]));  // no contraction: reproducible
    }
    uint64_t v = (uint64_t)frac;
    if (__dsub_rn(frac, (double)v) > 1.0 - 1e-9) v += 1;
    uint64_t *o = ext + (size_t)poly * (L + np) * n + (size_t)L * n + k;
    for (uint32_t kk = 0; kk < np; kk++) {
        const uint64_t *row = tab + (size_t)kk * (L + 1);  // qhat_i mod p_k (L values), Q mod p_k
        const PrimeConst p = pc[nq + kk];
        u128 a = {0, 0};
        for (uint32_t i = 0; i < L; i++) mac(a, yv[i], __ldg(row + i));
        o[(size_t)kk * n] = sub_mod(barrett(a, p), barrett(mul_wide(v, __ldg(row + L)), p), p.q);
    }
}

}  // namespace

// ------------------------------------------------------------------ host side

namespace {

struct ExtConsts {
    uint64_t *scale = nullptr;  // [L][4] inverse-NTT last-stage constants with qhat_i^-1 folded
    uint64_t *tab = nullptr;    // [np][L+1]
    double *qd = nullptr;       // [L] the primes as doubles
};

ExtConsts ext_consts(Context &c, uint32_t L) {
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.ext_consts.find(L);
    if (it != c.ext_consts.end())
        return ExtConsts{(uint64_t *)it->second[0], (uint64_t *)it->second[1], (double *)it->second[2]};
    ExtConsts e;
    std::vector<uint64_t> Q(c.primes.begin(), c.primes.begin() + L), sc, tab;
    std::vector<double> qi(L);
    for (uint32_t i = 0; i < L; i++) {
        uint64_t q = Q[i], h = host::partial_product(Q, i, q);
        uint64_t cc = host::mulmod(host::invmod(h, q), c.h_pc[i].n_inv, q);
        uint64_t psi_half_inv = 0;
        // psi^-(N/2) sits at index 1 of the inverse twiddle table
        SHM_CUDA(cudaMemcpy(&psi_half_inv, c.tw + (size_t)i * 4 * c.n + 2 * c.n + 1, 8, cudaMemcpyDeviceToHost));
        uint64_t c1 = host::mulmod(cc, psi_half_inv, q);
        sc.insert(sc.end(), {cc, host::shoup_of(cc, q), c1, host::shoup_of(c1, q)});
        qi[i] = (double)q;
    }
    for (uint32_t k = 0; k < c.np; k++) {
        uint64_t p = c.primes[c.nq + k], Qm = 1;
        for (uint32_t i = 0; i < L; i++) {
            tab.push_back(host::partial_product(Q, i, p));
            Qm = host::mulmod(Qm, Q[i] % p, p);
        }
        tab.push_back(Qm);
    }
    SHM_CUDA(cudaMalloc(&e.scale, sc.size() * 8));
    SHM_CUDA(cudaMemcpy(e.scale, sc.data(), sc.size() * 8, cudaMemcpyHostToDevice));
    SHM_CUDA(cudaMalloc(&e.tab, tab.size() * 8));
    SHM_CUDA(cudaMemcpy(e.tab, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice));
    SHM_CUDA(cudaMalloc(&e.qd, qi.size() * 8));
    SHM_CUDA(cudaMemcpy(e.qd, qi.data(), qi.size() * 8, cudaMemcpyHostToDevice));
    c.ext_consts[L] = {e.scale, e.tab, e.qd};
    return e;
}

}  // namespace

// The Sh-Rot / FmtSwitch inner products: groups are served in chunks that fit
// c.ip_chunk_bytes of shared memory, each chunk reading the key once.
void ip_multi(const Context &c, const uint64_t *up, const uint64_t *key, uint64_t *acc, uint32_t n_cts, uint32_t L,
              uint32_t beta, uint32_t H, const uint32_t *perm, cudaStream_t st) {
    static std::once_flag attr;
    std::call_once(attr, [] {
        for (const void *f : {(const void *)ip_multi_kernel<true>, (const void *)ip_multi_kernel<false>})
            SHM_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kIpSmemMax));
    });
    const uint32_t np = c.np, LP = L + np;
    const size_t cap = std::min<size_t>(c.ip_chunk_bytes, kIpSmemMax);
    const uint32_t chunk = std::max<uint32_t>(1, std::min<uint32_t>(n_cts, (uint32_t)(cap / (beta * kIpT * 8))));
    const dim3 grid(c.n / kIpT, LP, (n_cts + chunk - 1) / chunk);
    const size_t smem = (size_t)chunk * beta * kIpT * 8;
    SHM_LAUNCHED(1);
    if (c.s52)
        ip_multi_kernel<true><<<grid, kIpT, smem, st>>>(up, key, acc, n_cts, chunk, L, np, c.nq, beta, H, c.log_n,
                                                        c.pc, perm);
    else
        ip_multi_kernel<false><<<grid, kIpT, smem, st>>>(up, key, acc, n_cts, chunk, L, np, c.nq, beta, H, c.log_n,
                                                         c.pc, perm);
    SHM_CUDA(cudaGetLastError());
}

namespace {

void check_shape(const Context &c, uint32_t L, uint32_t beta, uint32_t H) {
    if (c.np == 0) throw std::invalid_argument("context has no special primes");
    if (L < 1 || L > c.nq) throw std::invalid_argument("level out of range");
    if (beta > (uint32_t)kMaxB || L + c.np > 64 || c.np > 16 || H < 2 || H > 64)
        throw std::invalid_argument("shared-a shape too large");
}

// inner products, ModDown and combine for one target; acc/delta are workspace
void apply_target(const Context &c, const uint64_t *up, uint32_t n_cts, uint32_t L, uint32_t beta, uint32_t H,
                  const Target &t, uint64_t *acc, uint64_t *delta, cudaStream_t st) {
    const uint32_t np = c.np, LP = L + np;
    ip_multi(c, up, t.key, acc, n_cts, L, beta, H, t.perm, st);
    LimbMap mp;
    for (uint32_t s = 0; s < 512; s++) mp.prime[s] = (s >= L && s < LP) ? (uint8_t)(c.nq + (s - L)) : 255;
    ntt_inverse(c, acc, n_cts * H * LP, LP, mp, c.moddown_scale, st, L);
    // conversion of the special-prime limbs, NTT and (acc - delta) P^-1 + sigma(add) fused
    ModDownIO md;
    md.acc = acc;
    md.conv = c.moddown_conv;
    md.pinv = c.p_inv;
    md.out = t.out;
    md.out_ct = (long long)t.out_ct;
    md.out_h = (long long)t.out_h;
    md.add = t.add;
    md.add_ct = (long long)t.add_ct;
    md.add_h = (long long)t.add_h;
    md.n_add = t.add ? t.n_add : 0;
    md.perm = t.perm;
    md.n_perm = md.n_add;
    md.H = H;
    md.np = np;
    md.s52 = c.s52 ? 1 : 0;
    ntt_forward_moddown(c, md, delta, n_cts * H, L, st);
}

}  // namespace

size_t shared_rotate_ws_words(const Context &c, uint32_t n_groups, uint32_t n, uint32_t L) {
    const uint32_t beta = (L + c.np - 1) / c.np, LP = L + c.np, H = n + 1;
    return (size_t)n_groups * c.n * (L + (size_t)beta * LP + (size_t)H * LP + (size_t)H * L);
}

void shared_rotate_hoisted(const Context &c, const uint64_t *sh, uint32_t n_groups, uint32_t n, uint32_t L,
                           uint32_t n_elts, const uint32_t *elts, const uint64_t *const *keys, uint64_t *const *outs,
                           uint64_t *ws, cudaStream_t st) {
    const uint32_t beta = (L + c.np - 1) / c.np, LP = L + c.np, H = n + 1;
    check_shape(c, L, beta, H);
    if (beta > c.dnum) throw std::invalid_argument("level needs more key digits than the key holds");
    const size_t ln = (size_t)L * c.n;
    uint64_t *x = ws, *up = x + (size_t)n_groups * ln, *acc = up + (size_t)n_groups * beta * LP * c.n;
    uint64_t *delta = acc + (size_t)n_groups * H * LP * c.n;
    modup_into(c, sh + (size_t)n * ln, (size_t)H * ln, n_groups, L, x, up, st);
    for (uint32_t e = 0; e < n_elts; e++) {
        Target t{keys[e], const_cast<Context &>(c).perm(elts[e]), outs[e], (size_t)H * ln, ln, sh, (size_t)H * ln,
                 ln, n};
        apply_target(c, up, n_groups, L, beta, H, t, acc, delta, st);
    }
}

size_t fmt_forward_ws_words(const Context &c, uint32_t n_groups, uint32_t n, uint32_t L) {
    const uint32_t LP = L + c.np, H = n + 1;
    return (size_t)n_groups * c.n * ((size_t)n * L + (size_t)n * LP + (size_t)H * LP + (size_t)H * L);
}

void fmt_forward(const Context &c, const uint64_t *cts, uint32_t n_groups, uint32_t n, uint32_t L,
                 const uint64_t *key, uint64_t *out, uint64_t *ws, cudaStream_t st) {
    const uint32_t LP = L + c.np, H = n + 1;
    check_shape(c, L, n, H);
    const size_t ln = (size_t)L * c.n, N = c.n;
    const uint32_t m = n_groups * n;  // member ciphertexts
    uint64_t *y = ws, *ext = y + (size_t)m * ln, *acc = ext + (size_t)m * LP * N;
    uint64_t *delta = acc + (size_t)n_groups * H * LP * N;
    ExtConsts e = ext_consts(const_cast<Context &>(c), L);
    // y = INTT(a_j) * qhat^-1 ; the Ql rows of ext keep a_j in NTT form
    SHM_CUDA(cudaMemcpy2DAsync(y, ln * 8, cts + ln, 2 * ln * 8, ln * 8, m, cudaMemcpyDeviceToDevice, st));
    ntt_inverse(c, y, m * L, L, q_map(L), e.scale, st);
    SHM_CUDA(cudaMemcpy2DAsync(ext, LP * N * 8, cts + ln, 2 * ln * 8, ln * 8, m, cudaMemcpyDeviceToDevice, st));
    SHM_LAUNCHED(1);
    exact_ext_kernel<<<dim3(N / kT, m), kT, 0, st>>>(y, ext, e.tab, e.qd, L, c.np, c.nq, c.log_n, c.pc);
    SHM_CUDA(cudaGetLastError());
    LimbMap mp;
    for (uint32_t s = 0; s < 512; s++) mp.prime[s] = (s >= L && s < LP) ? (uint8_t)(c.nq + (s - L)) : 255;
    ntt_forward(c, ext, m * LP, LP, mp, st);
    // digits = the n members of a group: ext is [G][n][LP][N]
    Target t{key, nullptr, out, (size_t)H * ln, ln, cts, (size_t)n * 2 * ln, 2 * ln, n};
    apply_target(c, ext, n_groups, L, n, H, t, acc, delta, st);
}

size_t fmt_backward_ws_words(const Context &c, uint32_t n_groups, uint32_t n, uint32_t L) {
    const uint32_t beta = (L + c.np - 1) / c.np, LP = L + c.np;
    (void)n;
    return (size_t)n_groups * c.n * (L + (size_t)beta * LP + 2 * (size_t)LP + 2 * (size_t)L);
}

void fmt_backward(const Context &c, const uint64_t *sh, uint32_t n_groups, uint32_t n, uint32_t L,
                  const uint64_t *const *keys, uint64_t *out, uint64_t *ws, cudaStream_t st) {
    const uint32_t beta = (L + c.np - 1) / c.np, LP = L + c.np, H = n + 1;
    check_shape(c, L, beta, 2);
    if (beta > c.dnum) throw std::invalid_argument("level needs more key digits than the key holds");
    const size_t ln = (size_t)L * c.n;
    uint64_t *x = ws, *up = x + (size_t)n_groups * ln, *acc = up + (size_t)n_groups * beta * LP * c.n;
    uint64_t *delta = acc + (size_t)n_groups * 2 * LP * c.n;
    modup_into(c, sh + (size_t)n * ln, (size_t)H * ln, n_groups, L, x, up, st);
    for (uint32_t i = 0; i < n; i++) {
        // member i of group g -> ordinary ciphertext g * n + i = (b_i + cx0, cx1)
        Target t{keys[i], nullptr, out + (size_t)i * 2 * ln, (size_t)n * 2 * ln, ln, sh + (size_t)i * ln,
                 (size_t)H * ln, 0, 1};
        apply_target(c, up, n_groups, L, beta, 2, t, acc, delta, st);
    }
}

// ------------------------------------------------------------------ extended basis QlP

namespace {

// out[row][j] = P * in[row][j] mod q_j for j < L, 0 for the special-prime limbs.  Grid (N/kT, LP, rows)
__global__ void extend_kernel(const uint64_t *__restrict__ in, uint64_t *__restrict__ out, uint32_t L, uint32_t np,
                              uint32_t log_n, const PrimeConst *__restrict__ pc, const uint64_t *__restrict__ pmod) {
    const uint32_t j = blockIdx.y, row = blockIdx.z, LP = L + np;
    const uint32_t k = blockIdx.x * kT + threadIdx.x;
    uint64_t v = 0;
    if (j < L) v = shoup(in[(((size_t)row * L + j) << log_n) + k], pmod[2 * j], pmod[2 * j + 1], pc[j].q);
    out[(((size_t)row * LP + j) << log_n) + k] = v;
}

// rows of LP limbs, limb j under prime j (j < L) or the special prime nq + j - L.  Grid (N/kT, LP, rows)
__global__ void add_ext_kernel(const uint64_t *__restrict__ a, const uint64_t *__restrict__ b, uint64_t *__restrict__ out,
                               uint32_t L, uint32_t np, uint32_t nq, uint32_t log_n, const PrimeConst *__restrict__ pc) {
    const uint32_t j = blockIdx.y, row = blockIdx.z, LP = L + np;
    const size_t off = (((size_t)row * LP + j) << log_n) + blockIdx.x * kT + threadIdx.x;
    out[off] = add_mod(a[off], b[off], pc[j < L ? j : nq + (j - L)].q);
}

// The extended Sh-Rot output of one target: out[g][h] = acc[g][h] (+ for the b rows h < n the
// rotated b: over every limb sigma(b_ext) when the input is extended, else P sigma(b) on the
// Q limbs).  Grid (N/kT, LP, groups * H)
__global__ void combine_ext_kernel(const uint64_t *__restrict__ acc, uint64_t *__restrict__ out,
                                   const uint64_t *__restrict__ bsrc, int b_ext, const uint32_t *__restrict__ perm,
                                   uint32_t H, uint32_t L, uint32_t np, uint32_t nq, uint32_t log_n,
                                   const PrimeConst *__restrict__ pc, const uint64_t *__restrict__ pmod) {
    const uint32_t j = blockIdx.y, gh = blockIdx.z, h = gh % H, LP = L + np;
    const uint32_t k = blockIdx.x * kT + threadIdx.x;
    const size_t off = (((size_t)gh * LP + j) << log_n) + k;
    uint64_t v = acc[off];
    if (h + 1 < H) {
        const uint32_t ks = perm ? __ldg(perm + k) : k;
        const uint64_t q = pc[j < L ? j : nq + (j - L)].q;
        if (b_ext)
            v = add_mod(v, bsrc[(((size_t)gh * LP + j) << log_n) + ks], q);
        else if (j < L)
            v = add_mod(v, shoup(bsrc[(((size_t)gh * L + j) << log_n) + ks], pmod[2 * j], pmod[2 * j + 1], q), q);
    }
    out[off] = v;
}

// ModDown of n_polys extended polynomials (their special-prime limbs are overwritten by the
// inverse NTT) into out [n_polys][L][N]; delta: [n_polys][L][N] scratch
void moddown_rows(const Context &c, uint64_t *ext, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t *delta,
                  cudaStream_t st) {
    const uint32_t LP = L + c.np;
    LimbMap mp;
    for (uint32_t s = 0; s < 512; s++) mp.prime[s] = (s >= L && s < LP) ? (uint8_t)(c.nq + (s - L)) : 255;
    ntt_inverse(c, ext, n_polys * LP, LP, mp, c.moddown_scale, st, L);
    ModDownIO md;
    md.acc = ext;
    md.conv = c.moddown_conv;
    md.pinv = c.p_inv;
    md.out = out;
    md.out_ct = (long long)L * c.n;
    md.H = 1;
    md.np = c.np;
    md.s52 = c.s52 ? 1 : 0;
    ntt_forward_moddown(c, md, delta, n_polys, L, st);
}

}  // namespace

LimbMap ext_map(uint32_t L, const Context &c) {
    LimbMap m;
    for (uint32_t s = 0; s < 512; s++) m.prime[s] = s < L ? (uint8_t)s : (s < L + c.np ? (uint8_t)(c.nq + (s - L)) : 255);
    return m;
}

void extend(const Context &c, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L, cudaStream_t st) {
    if (!n_polys) return;
    SHM_LAUNCHED(1);
    extend_kernel<<<dim3(c.n / kT, L + c.np, n_polys), kT, 0, st>>>(in, out, L, c.np, c.log_n, c.pc, c.p_mod);
    SHM_CUDA(cudaGetLastError());
}

void add_ext(const Context &c, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys, uint32_t L,
             cudaStream_t st) {
    if (!n_polys) return;
    SHM_LAUNCHED(1);
    add_ext_kernel<<<dim3(c.n / kT, L + c.np, n_polys), kT, 0, st>>>(a, b, out, L, c.np, c.nq, c.log_n, c.pc);
    SHM_CUDA(cudaGetLastError());
}

size_t moddown_ext_ws_words(const Context &c, uint32_t n_polys, uint32_t L) { return (size_t)n_polys * L * c.n; }

void moddown_ext(const Context &c, uint64_t *ext, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t *ws,
                 cudaStream_t st) {
    if (!n_polys) return;
    if (c.np == 0) throw std::invalid_argument("context has no special primes");
    moddown_rows(c, ext, out, n_polys, L, ws, st);
}

size_t shared_rotate_ext_ws_words(const Context &c, uint32_t n_groups, uint32_t n, uint32_t L) {
    const uint32_t beta = (L + c.np - 1) / c.np, LP = L + c.np, H = n + 1;
    // x, up, acc, the a rows (extended input), their ModDown and its delta
    return (size_t)n_groups * c.n * (L + (size_t)beta * LP + (size_t)H * LP + LP + 2 * (size_t)L);
}

void shared_rotate_ext(const Context &c, const uint64_t *in, bool in_ext, uint32_t n_groups, uint32_t n, uint32_t L,
                       uint32_t n_elts, const uint32_t *elts, const uint64_t *const *keys, uint64_t *const *outs,
                       uint64_t *ws, cudaStream_t st) {
    const uint32_t beta = (L + c.np - 1) / c.np, LP = L + c.np, H = n + 1;
    check_shape(c, L, beta, H);
    if (beta > c.dnum) throw std::invalid_argument("level needs more key digits than the key holds");
    const size_t N = c.n, ln = (size_t)L * N;
    uint64_t *x = ws, *up = x + (size_t)n_groups * ln, *acc = up + (size_t)n_groups * beta * LP * N;
    uint64_t *arow = acc + (size_t)n_groups * H * LP * N, *aq = arow + (size_t)n_groups * LP * N;
    uint64_t *delta = aq + (size_t)n_groups * ln;
    const size_t g_words = (size_t)H * (in_ext ? LP : L) * N;  // one input group
    if (in_ext) {
        // ModDown of the a row of every group, then ModUp of it
        SHM_CUDA(cudaMemcpy2DAsync(arow, LP * N * 8, in + (size_t)n * LP * N, g_words * 8, LP * N * 8, n_groups,
                                   cudaMemcpyDeviceToDevice, st));
        moddown_rows(c, arow, aq, n_groups, L, delta, st);
        modup_into(c, aq, ln, n_groups, L, x, up, st);
    } else {
        modup_into(c, in + (size_t)n * ln, g_words, n_groups, L, x, up, st);
    }
    for (uint32_t e = 0; e < n_elts; e++) {
        const uint32_t *perm = const_cast<Context &>(c).perm(elts[e]);
        ip_multi(c, up, keys[e], acc, n_groups, L, beta, H, perm, st);
        SHM_LAUNCHED(1);
        combine_ext_kernel<<<dim3(N / kT, LP, n_groups * H), kT, 0, st>>>(acc, outs[e], in, in_ext ? 1 : 0, perm, H, L,
                                                                          c.np, c.nq, c.log_n, c.pc, c.p_mod);
        SHM_CUDA(cudaGetLastError());
    }
}

}  // namespace shm
