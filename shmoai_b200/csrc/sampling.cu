// Counter-based sampling (key generation, encryption) and the signed-coefficient lift.
//
// Every value is a pure function of (seed, index): splitmix64's output mix applied to
// seed + index * golden gamma (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014).  The same function in the CPU restatement gives the same
// keys and ciphertexts bit for bit, which is what lets a whole pipeline be compared
// between the two.  The distributions are those of the reference's samplers
// (thirdparty/phantom-fhe/src/prng.cu:142-240): uniform residues mod each prime and a
// centred binomial over 21 + 21 bits (sigma ~ 3.24); the streams are not.
#include "core.hpp"

namespace shm {

namespace {

constexpr int kT = 256;

__device__ __forceinline__ uint64_t mix64(uint64_t seed, uint64_t idx) {
    uint64_t z = seed + (idx + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// out[p][i][k] = floor((h1 * 2^64 + h2) * q_i / 2^128), h1, h2 the two hashes of (p, i, k)
__global__ void uniform_kernel(uint64_t *__restrict__ out, uint32_t L, uint32_t log_n, uint64_t seed,
                               const PrimeConst *__restrict__ pc) {
    const uint32_t row = blockIdx.y;  // p * L + i
    const uint32_t k = blockIdx.x * kT + threadIdx.x;
    const uint64_t q = pc[row % L].q;
    const uint64_t idx = ((uint64_t)row << log_n) + k;
    const uint64_t h1 = mix64(seed, 2 * idx), h2 = mix64(seed, 2 * idx + 1);
    const uint64_t lo_hi = __umul64hi(h2, q);
    const uint64_t lo = h1 * q, hi = __umul64hi(h1, q);
    const uint64_t s = lo + lo_hi;
    out[((size_t)row << log_n) + k] = hi + (s < lo ? 1 : 0);
}

// one centred-binomial integer per (p, k), written as residues mod each of the L primes
__global__ void cbd_kernel(uint64_t *__restrict__ out, uint32_t L, uint32_t log_n, uint64_t seed,
                           const PrimeConst *__restrict__ pc) {
    const uint32_t p = blockIdx.y;
    const uint32_t k = blockIdx.x * kT + threadIdx.x;
    const uint64_t h = mix64(seed, ((uint64_t)p << log_n) + k);
    const int e = __popcll(h & 0x1FFFFFull) - __popcll((h >> 21) & 0x1FFFFFull);
    uint64_t *o = out + ((size_t)p * L << log_n) + k;
    for (uint32_t i = 0; i < L; i++) {
        const uint64_t q = pc[i].q;
        o[(size_t)i << log_n] = e >= 0 ? (uint64_t)e : q - (uint64_t)(-e);
    }
}

// rows of L limbs; limb i < Lq uses prime i, limb i >= Lq the special prime nq + i - Lq
__global__ void lift_kernel(const int64_t *__restrict__ in, uint64_t *__restrict__ out, uint32_t L, uint32_t log_n,
                            const PrimeConst *__restrict__ pc, uint32_t Lq, uint32_t nq) {
    const uint32_t p = blockIdx.y;
    const uint32_t k = blockIdx.x * kT + threadIdx.x;
    const int64_t v = in[((size_t)p << log_n) + k];
    const uint64_t mag = v < 0 ? (uint64_t)(-(v + 1)) + 1 : (uint64_t)v;  // |v| without overflow
    uint64_t *o = out + ((size_t)p * L << log_n) + k;
    for (uint32_t i = 0; i < L; i++) {
        const uint64_t q = pc[i < Lq ? i : nq + (i - Lq)].q, r = mag % q;
        o[(size_t)i << log_n] = (v < 0 && r) ? q - r : r;
    }
}

}  // namespace

void sample_uniform(const Context &c, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t seed, cudaStream_t st) {
    if (!n_polys) return;
    SHM_LAUNCHED(1);
    uniform_kernel<<<dim3(c.n / kT, n_polys * L), kT, 0, st>>>(out, L, c.log_n, seed, c.pc);
    SHM_CUDA(cudaGetLastError());
}

void sample_cbd(const Context &c, uint64_t *out, uint32_t n_polys, uint32_t L, uint64_t seed, cudaStream_t st) {
    if (!n_polys) return;
    SHM_LAUNCHED(1);
    cbd_kernel<<<dim3(c.n / kT, n_polys), kT, 0, st>>>(out, L, c.log_n, seed, c.pc);
    SHM_CUDA(cudaGetLastError());
}

void lift_signed(const Context &c, const int64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L, cudaStream_t st) {
    if (!n_polys) return;
    SHM_LAUNCHED(1);
    lift_kernel<<<dim3(c.n / kT, n_polys), kT, 0, st>>>(in, out, L, c.log_n, c.pc, L, c.nq);
    SHM_CUDA(cudaGetLastError());
}

void lift_signed_ext(const Context &c, const int64_t *in, uint64_t *out, uint32_t n_polys, uint32_t L,
                     cudaStream_t st) {
    if (!n_polys) return;
    SHM_LAUNCHED(1);
    lift_kernel<<<dim3(c.n / kT, n_polys), kT, 0, st>>>(in, out, L + c.np, c.log_n, c.pc, L, c.nq);
    SHM_CUDA(cudaGetLastError());
}

}  // namespace shm
