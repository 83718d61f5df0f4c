// Kernels used by the bootstrapping pipeline and the scale-exact evaluator:
// per-limb scalar multiply / add, multiply-plain-accumulate (the inner sums of
// the baby-step giant-step linear transforms), the mod-raise lift and the
// limb drop.
//
// Reference counterparts: multiply_const / add_const in the moai adapter
// (src/include/source/ckks_evaluator_parallel.cuh:245-280), the per-diagonal
// multiply_plain + add_inplace of Bootstrapper::bsgs_linear_transform
// (src/include/source/bootstrapping/Bootstrapper.cu:2168-2340) and
// Bootstrapper::modraise_inplace (Bootstrapper.cu:3271-3356: centred lift of
// the q0 limb into every prime).
#include "core.hpp"

namespace shm {

namespace {

constexpr int kT = 256;

// out[row] = a[row] * s[limb] (Shoup), rows = n_polys * L
__global__ void mul_scalar_kernel(const uint64_t *__restrict__ a, uint64_t *__restrict__ out, ScalarTab s, uint32_t L,
                                  uint32_t log_n, const PrimeConst *__restrict__ pc) {
    const uint32_t row = blockIdx.y, limb = row % L;
    const uint64_t q = pc[limb].q, w = s.v[limb], ws = s.shoup[limb];
    const size_t off = ((size_t)row << log_n) + 2 * (blockIdx.x * kT + threadIdx.x);
    ulonglong2 x = *reinterpret_cast<const ulonglong2 *>(a + off);
    x.x = shoup(x.x, w, ws, q);
    x.y = shoup(x.y, w, ws, q);
    *reinterpret_cast<ulonglong2 *>(out + off) = x;
}

// c0 rows of every ciphertext get + s[limb]; c1 rows are copied
__global__ void add_scalar_kernel(const uint64_t *__restrict__ a, uint64_t *__restrict__ out, ScalarTab s, uint32_t L,
                                  uint32_t log_n, const PrimeConst *__restrict__ pc) {
    const uint32_t row = blockIdx.y, limb = row % L, poly = (row / L) & 1;
    const size_t off = ((size_t)row << log_n) + 2 * (blockIdx.x * kT + threadIdx.x);
    ulonglong2 x = *reinterpret_cast<const ulonglong2 *>(a + off);
    if (poly == 0) {
        const uint64_t q = pc[limb].q, c = s.v[limb];
        x.x = add_mod(x.x, c, q);
        x.y = add_mod(x.y, c, q);
    }
    *reinterpret_cast<ulonglong2 *>(out + off) = x;
}

// out[c] = sum_t X_t[c] * P_t   over k terms (X_t: [n_polys][L][N], P_t: [L][N])
// Limb-major block order: blockIdx.y = limb * n_polys + poly, so the polynomials that share a
// plaintext limb run together and the k plaintext limbs stay in L2 for all of them.
// L = limbs per row; limb l uses prime l when l < Lq, else the special prime nq + l - Lq
__global__ void mul_plain_acc_kernel(PtrTab X, PtrTab P, uint32_t k, uint64_t *__restrict__ out, uint32_t L,
                                     uint32_t log_n, const PrimeConst *__restrict__ pc, int accumulate, uint32_t Lq,
                                     uint32_t nq) {
    const uint32_t n_polys = gridDim.y / L, limb = blockIdx.y / n_polys, row = (blockIdx.y % n_polys) * L + limb;
    const PrimeConst p = pc[limb < Lq ? limb : nq + (limb - Lq)];
    const size_t off = ((size_t)row << log_n) + blockIdx.x * kT + threadIdx.x;
    const size_t poff = ((size_t)limb << log_n) + blockIdx.x * kT + threadIdx.x;
    u128 acc = {0, 0};
    // unrolled so that a group of terms' loads is in flight together (the loads, not the
    // multiplies, bound this kernel)
#pragma unroll 8
    for (uint32_t t = 0; t < k; t++) mac(acc, X.p[t][off], P.p[t][poff]);
    uint64_t r = barrett(acc, p);
    if (accumulate) r = add_mod(r, out[off], p.q);
    out[off] = r;
}

// out[ct][p][limb] = sum_t w_t[limb] X_t[ct][p][limb] (+ w0[limb] for p = 0); each lazy Shoup
// product is below 2q and the running sum is kept below 4q (one conditional subtraction
// per term), so the sum stays below 5q < 2^(k+7) for every prime below 2^61 and one
// reduce_small finishes it.  Grid (N/2/256, L, 2 n_cts).
__global__ void lin_comb_kernel(LinTerms t, uint64_t *__restrict__ out, uint32_t L, uint32_t log_n,
                                const PrimeConst *__restrict__ pc) {
    const uint32_t limb = blockIdx.y, poly = blockIdx.z, ct = poly >> 1, p = poly & 1;
    const PrimeConst pr = pc[limb];
    const size_t col = 2 * (blockIdx.x * kT + threadIdx.x);
    uint64_t a0 = 0, a1 = 0;
    for (uint32_t i = 0; i < t.k; i++) {
        const size_t off = ((((size_t)ct * 2 + p) * t.levels[i] + limb) << log_n) + col;
        const ulonglong2 x = *reinterpret_cast<const ulonglong2 *>(t.x[i] + off);
        a0 = csub(a0 + shoup_lazy(x.x, t.w[i][limb], t.ws[i][limb], pr.q), 2 * pr.q);
        a1 = csub(a1 + shoup_lazy(x.y, t.w[i][limb], t.ws[i][limb], pr.q), 2 * pr.q);
    }
    if (p == 0 && t.has_w0) {
        a0 += t.w0[limb];
        a1 += t.w0[limb];
    }
    ulonglong2 r;
    r.x = reduce_small(a0, pr);
    r.y = reduce_small(a1, pr);
    *reinterpret_cast<ulonglong2 *>(out + ((((size_t)ct * 2 + p) * L + limb) << log_n) + col) = r;
}

// t_j = centred lift of c (mod q0) into prime j, for j < L
__global__ void modraise_spread(const uint64_t *__restrict__ c0, uint64_t *__restrict__ out, uint32_t L,
                                uint32_t log_n, const PrimeConst *__restrict__ pc) {
    const uint32_t j = blockIdx.y, poly = blockIdx.z;
    const uint32_t k = blockIdx.x * kT + threadIdx.x;
    const uint64_t q0 = pc[0].q;
    const uint64_t v = c0[((size_t)poly << log_n) + k];
    const PrimeConst p = pc[j];
    uint64_t r = barrett({v, 0}, p);
    if (v > (q0 >> 1)) r = sub_mod(r, barrett({q0, 0}, p), p.q);
    out[(((size_t)poly * L + j) << log_n) + k] = r;
}

}  // namespace

void mul_scalar(const Context &c, const uint64_t *a, uint64_t *out, const ScalarTab &s, uint32_t n_polys, uint32_t L,
                cudaStream_t st) {
    if (!n_polys) return;
    SHM_LAUNCHED(1);
    mul_scalar_kernel<<<dim3(c.n / 2 / kT, n_polys * L), kT, 0, st>>>(a, out, s, L, c.log_n, c.pc);
    SHM_CUDA(cudaGetLastError());
}

void add_scalar(const Context &c, const uint64_t *a, uint64_t *out, const ScalarTab &s, uint32_t n_cts, uint32_t L,
                cudaStream_t st) {
    if (!n_cts) return;
    SHM_LAUNCHED(1);
    add_scalar_kernel<<<dim3(c.n / 2 / kT, n_cts * 2 * L), kT, 0, st>>>(a, out, s, L, c.log_n, c.pc);
    SHM_CUDA(cudaGetLastError());
}

void mul_plain_acc(const Context &c, const PtrTab &X, const PtrTab &P, uint32_t k, uint64_t *out, uint32_t n_polys,
                   uint32_t L, bool accumulate, cudaStream_t st, bool ext) {
    if (!n_polys || !k) return;
    const uint32_t rows = ext ? L + c.np : L;
    SHM_LAUNCHED(1);
    mul_plain_acc_kernel<<<dim3(c.n / kT, n_polys * rows), kT, 0, st>>>(X, P, k, out, rows, c.log_n, c.pc,
                                                                         accumulate ? 1 : 0, L, c.nq);
    SHM_CUDA(cudaGetLastError());
}

void linear_combination(const Context &c, const LinTerms &t, uint64_t *out, uint32_t n_cts, uint32_t L,
                        cudaStream_t st) {
    if (!n_cts) return;
    if (t.k < 1 || t.k > (uint32_t)kMaxLinTerms) throw std::invalid_argument("linear combination of 1..8 terms");
    if (L < 1 || L > 64) throw std::invalid_argument("level out of range");
    for (uint32_t i = 0; i < t.k; i++)
        if (t.levels[i] < L) throw std::invalid_argument("a term has fewer limbs than the result");
    SHM_LAUNCHED(1);
    lin_comb_kernel<<<dim3(c.n / 2 / kT, L, 2 * n_cts), kT, 0, st>>>(t, out, L, c.log_n, c.pc);
    SHM_CUDA(cudaGetLastError());
}

void modraise(const Context &c, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t *ws,
              cudaStream_t st) {
    // limb 0 of each polynomial (already contiguous when the input has one limb)
    SHM_CUDA(cudaMemcpyAsync(ws, in, (size_t)n_polys * c.n * 8, cudaMemcpyDeviceToDevice, st));
    LimbMap m;
    for (int i = 0; i < 512; i++) m.prime[i] = 255;
    m.prime[0] = 0;
    ntt_inverse(c, ws, n_polys, 1, m, nullptr, st);
    SHM_LAUNCHED(1);
    modraise_spread<<<dim3(c.n / kT, L, n_polys), kT, 0, st>>>(ws, out, L, c.log_n, c.pc);
    SHM_CUDA(cudaGetLastError());
    ntt_forward(c, out, n_polys * L, L, q_map(L), st);
}

}  // namespace shm
