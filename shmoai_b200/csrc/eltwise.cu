// Element-wise RNS kernels: add / sub / negate / multiply_plain, the 2x2 tensor
// product, NTT-domain automorphisms and the floor rescale.
//
// Reference semantics: thirdparty/phantom-fhe/src/polymath.cu:17-230 (pointwise mod q),
// :468-504 (tensor), src/galois.cu:8-21 (NTT-domain permutation),
// src/rns.cu:1125-1181 (rescale = (c_j - NTT(c_last mod q_j)) * q_last^-1, floor).
#include "core.hpp"

namespace shm {

namespace {

constexpr int kEwThreads = 256;

// Grid: (N/2/256 chunks) x rows; each thread handles 2 consecutive words of one limb.
template <EwOp OP>
__global__ void ew_kernel(const uint64_t *__restrict__ a, const uint64_t *__restrict__ b, uint64_t *__restrict__ out,
                          uint32_t L, uint32_t log_n, uint32_t b_polys, const PrimeConst *__restrict__ pc) {
    const uint32_t row = blockIdx.y;
    const uint32_t limb = row % L;
    const PrimeConst p = pc[limb];
    const size_t off = ((size_t)row << log_n) + 2 * (blockIdx.x * kEwThreads + threadIdx.x);
    const size_t boff = ((size_t)((row / L) % b_polys * L + limb) << log_n) + 2 * (blockIdx.x * kEwThreads + threadIdx.x);
    ulonglong2 x = *reinterpret_cast<const ulonglong2 *>(a + off), r;
    if constexpr (OP == EwOp::Negate) {
        r.x = x.x ? p.q - x.x : 0;
        r.y = x.y ? p.q - x.y : 0;
    } else {
        ulonglong2 y = *reinterpret_cast<const ulonglong2 *>(b + boff);
        if constexpr (OP == EwOp::Add) {
            r.x = add_mod(x.x, y.x, p.q);
            r.y = add_mod(x.y, y.y, p.q);
        } else if constexpr (OP == EwOp::Sub) {
            r.x = sub_mod(x.x, y.x, p.q);
            r.y = sub_mod(x.y, y.y, p.q);
        } else {
            r.x = mul_mod(x.x, y.x, p);
            r.y = mul_mod(x.y, y.y, p);
        }
    }
    *reinterpret_cast<ulonglong2 *>(out + off) = r;
}

// out[ct][p] = a[ct][p] + (p < sb ? b[ct][p] : 0); rows ct * sa * L + p * L + limb
__global__ void add_sizes_kernel(const uint64_t *__restrict__ a, const uint64_t *__restrict__ b,
                                 uint64_t *__restrict__ out, uint32_t sa, uint32_t sb, uint32_t L, uint32_t log_n,
                                 const PrimeConst *__restrict__ pc) {
    const uint32_t row = blockIdx.y, limb = row % L, p = (row / L) % sa, ct = row / (L * sa);
    const size_t col = 2 * (blockIdx.x * kEwThreads + threadIdx.x);
    const size_t off = ((size_t)row << log_n) + col;
    ulonglong2 x = *reinterpret_cast<const ulonglong2 *>(a + off);
    if (p < sb) {
        const size_t boff = (((size_t)(ct * sb + p) * L + limb) << log_n) + col;
        const ulonglong2 y = *reinterpret_cast<const ulonglong2 *>(b + boff);
        const uint64_t q = pc[limb].q;
        x.x = add_mod(x.x, y.x, q);
        x.y = add_mod(x.y, y.y, q);
    }
    *reinterpret_cast<ulonglong2 *>(out + off) = x;
}

// (a0, a1) x (b0, b1) -> (a0 b0, a0 b1 + a1 b0, a1 b1) per ciphertext
__global__ void tensor_kernel(const uint64_t *__restrict__ a, const uint64_t *__restrict__ b, uint64_t *__restrict__ out,
                              uint32_t L, uint32_t log_n, const PrimeConst *__restrict__ pc) {
    const uint32_t limb = blockIdx.y, ct = blockIdx.z;
    const PrimeConst p = pc[limb];
    const size_t ln = (size_t)L << log_n;
    const size_t k = ((size_t)limb << log_n) + blockIdx.x * kEwThreads + threadIdx.x;
    const uint64_t *A = a + ct * 2 * ln, *B = b + ct * 2 * ln;
    uint64_t *O = out + ct * 3 * ln;
    uint64_t a0 = A[k], a1 = A[ln + k], b0 = B[k], b1 = B[ln + k];
    O[k] = mul_mod(a0, b0, p);
    u128 m = mul_wide(a0, b1);
    mac(m, a1, b0);
    O[ln + k] = barrett(m, p);
    O[2 * ln + k] = mul_mod(a1, b1, p);
}

// out[ct] (+)= sum_{t < k} A_t[ct a_step] x B_t[ct b_step]: the size-3 tensor products of k
// ciphertext pairs summed before one reduction (step 0 broadcasts one ciphertext over the batch).
// The host bounds k so that each sum (2k products for the middle term) stays below the Barrett
// bound; S52: the products' 32-bit partials summed in three 64-bit words (every prime < 2^52).
template <bool S52>
__global__ void tensor_acc_kernel(PtrTab A, PtrTab B, uint32_t k, uint32_t a_step, uint32_t b_step,
                                  uint64_t *__restrict__ out, uint32_t L, uint32_t log_n,
                                  const PrimeConst *__restrict__ pc, int accumulate) {
    const uint32_t limb = blockIdx.y, ct = blockIdx.z;
    const PrimeConst p = pc[limb];
    const size_t ln = (size_t)L << log_n;
    const size_t kk = ((size_t)limb << log_n) + blockIdx.x * kEwThreads + threadIdx.x;
    Acc<S52> s0, s1, s2;
    for (uint32_t t = 0; t < k; t++) {
        const uint64_t *a = A.p[t] + (size_t)ct * a_step * 2 * ln, *b = B.p[t] + (size_t)ct * b_step * 2 * ln;
        const uint64_t a0 = a[kk], a1 = a[ln + kk], b0 = b[kk], b1 = b[ln + kk];
        s0.add(a0, b0);
        s1.add(a0, b1);
        s1.add(a1, b0);
        s2.add(a1, b1);
    }
    uint64_t *O = out + (size_t)ct * 3 * ln;
    uint64_t r0 = barrett(s0.get(), p), r1 = barrett(s1.get(), p), r2 = barrett(s2.get(), p);
    if (accumulate) {
        r0 = add_mod(r0, O[kk], p.q);
        r1 = add_mod(r1, O[ln + kk], p.q);
        r2 = add_mod(r2, O[2 * ln + kk], p.q);
    }
    O[kk] = r0;
    O[ln + kk] = r1;
    O[2 * ln + kk] = r2;
}

// NTT-domain automorphism computed per element: slot k takes slot perm(k) with
// 2 brv(perm(k)) + 1 = (2 brv(k) + 1) elt mod 2N (the table of Context::perm, without the table)
__global__ void galois_kernel(const uint64_t *__restrict__ in, uint64_t *__restrict__ out, uint32_t elt,
                              uint32_t log_n) {
    const size_t row = blockIdx.y;
    const uint32_t k = blockIdx.x * kEwThreads + threadIdx.x;
    out[(row << log_n) + k] = in[(row << log_n) + galois_index(k, elt, log_n)];
}

// copy the last limb of every polynomial into a contiguous buffer
__global__ void gather_last(const uint64_t *__restrict__ in, uint64_t *__restrict__ last, uint32_t L, uint32_t log_n) {
    const uint32_t poly = blockIdx.y;
    const uint32_t k = blockIdx.x * kEwThreads + threadIdx.x;
    last[((size_t)poly << log_n) + k] = in[(((size_t)poly * L + L - 1) << log_n) + k];
}

}  // namespace

void elementwise(const Context &c, EwOp op, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_polys,
                 uint32_t L, uint32_t b_polys, cudaStream_t st) {
    if (n_polys == 0 || L == 0) return;
    dim3 grid(c.n / 2 / kEwThreads, n_polys * L);
    if (b_polys == 0) b_polys = n_polys;
    switch (op) {
        case EwOp::Add: SHM_LAUNCHED(1); ew_kernel<EwOp::Add><<<grid, kEwThreads, 0, st>>>(a, b, out, L, c.log_n, b_polys, c.pc); break;
        case EwOp::Sub: SHM_LAUNCHED(1); ew_kernel<EwOp::Sub><<<grid, kEwThreads, 0, st>>>(a, b, out, L, c.log_n, b_polys, c.pc); break;
        case EwOp::Negate:
            SHM_LAUNCHED(1); ew_kernel<EwOp::Negate><<<grid, kEwThreads, 0, st>>>(a, b, out, L, c.log_n, b_polys, c.pc);
            break;
        case EwOp::MulPlain:
            SHM_LAUNCHED(1); ew_kernel<EwOp::MulPlain><<<grid, kEwThreads, 0, st>>>(a, b, out, L, c.log_n, b_polys, c.pc);
            break;
    }
    SHM_CUDA(cudaGetLastError());
}

void add_sizes(const Context &c, const uint64_t *a, uint32_t sa, const uint64_t *b, uint32_t sb, uint64_t *out,
               uint32_t n_cts, uint32_t L, cudaStream_t st) {
    if (n_cts == 0 || L == 0) return;
    if (sb > sa || sb == 0) throw std::invalid_argument("add_sizes: need a_size >= b_size >= 1");
    if ((size_t)n_cts * sa * L > 65535) throw std::invalid_argument("add_sizes: batch too large for one launch");
    SHM_LAUNCHED(1);
    add_sizes_kernel<<<dim3(c.n / 2 / kEwThreads, n_cts * sa * L), kEwThreads, 0, st>>>(a, b, out, sa, sb, L, c.log_n,
                                                                                         c.pc);
    SHM_CUDA(cudaGetLastError());
}

void tensor(const Context &c, const uint64_t *a, const uint64_t *b, uint64_t *out, uint32_t n_cts, uint32_t L,
            cudaStream_t st) {
    if (n_cts == 0) return;
    SHM_LAUNCHED(1); tensor_kernel<<<dim3(c.n / kEwThreads, L, n_cts), kEwThreads, 0, st>>>(a, b, out, L, c.log_n, c.pc);
    SHM_CUDA(cudaGetLastError());
}

void tensor_accumulate(const Context &c, const PtrTab &A, const PtrTab &B, uint32_t k, uint32_t a_step,
                       uint32_t b_step, uint64_t *out, uint32_t n_cts, uint32_t L, bool accumulate, cudaStream_t st) {
    if (n_cts == 0 || k == 0) return;
    const dim3 grid(c.n / kEwThreads, L, n_cts);
    SHM_LAUNCHED(1);
    if (c.s52)
        tensor_acc_kernel<true><<<grid, kEwThreads, 0, st>>>(A, B, k, a_step, b_step, out, L, c.log_n, c.pc,
                                                             accumulate ? 1 : 0);
    else
        tensor_acc_kernel<false><<<grid, kEwThreads, 0, st>>>(A, B, k, a_step, b_step, out, L, c.log_n, c.pc,
                                                              accumulate ? 1 : 0);
    SHM_CUDA(cudaGetLastError());
}

void apply_galois(const Context &c, const uint64_t *in, uint64_t *out, uint32_t rows, uint32_t elt, cudaStream_t st) {
    if (rows == 0) return;
    SHM_LAUNCHED(1); galois_kernel<<<dim3(c.n / kEwThreads, rows), kEwThreads, 0, st>>>(in, out, elt, c.log_n);
    SHM_CUDA(cudaGetLastError());
}

size_t rescale_ws_words(const Context &c, uint32_t n_polys, uint32_t L) {
    return (size_t)n_polys * L * c.n;  // last limbs (n_polys) + spread (n_polys * (L-1))
}

void rescale(const Context &c, const uint64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t *ws,
             cudaStream_t st) {
    if (L < 2) throw std::invalid_argument("rescale needs at least two limbs");
    if (n_polys == 0) return;  // nothing to do; a grid with y = 0 would be an invalid launch
    uint64_t *last = ws, *t = ws + ((size_t)n_polys << c.log_n);
    const uint32_t chunks = c.n / kEwThreads;
    SHM_LAUNCHED(1); gather_last<<<dim3(chunks, n_polys), kEwThreads, 0, st>>>(in, last, L, c.log_n);
    SHM_CUDA(cudaGetLastError());
    LimbMap m;
    for (int i = 0; i < 512; i++) m.prime[i] = 255;
    m.prime[0] = (uint8_t)(L - 1);
    ntt_inverse(c, last, n_polys, 1, m, nullptr, st);
    // t_j = c_last mod q_j, its NTT and out_j = (c_j - t_j) q_last^-1 in one NTT launch pair
    RescaleIO io;
    io.last = last;
    io.in = in;
    io.out = out;
    io.inv = c.rescale_inv + 2 * (size_t)(L - 1) * c.nq;
    ntt_forward_rescale(c, io, t, n_polys, L, st);
}

}  // namespace shm
