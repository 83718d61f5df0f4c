// Device modular arithmetic for word-size primes q < 2^62.
//
// * Shoup multiplication by a fixed operand w (w' = floor(w * 2^64 / q)):
//   one mul.hi + two mul.lo, result in [0, 2q).
// * Barrett reduction of a 128-bit value x < 2^(63+k) for a k-bit q:
//   t = x >> (k-1), qhat = mulhi(t, mu) with mu = floor(2^(63+k) / q),
//   r = x - qhat*q lies in [0, 3q); two conditional subtractions finish.
//   The bound x < 2^(63+k) admits sums of up to 2^(63-k) products a*b
//   (a, b < q), which is what the base conversions and the key-switching
//   inner product accumulate.
#pragma once
#include <cstdint>

namespace shm {

struct PrimeConst {
    uint64_t q;      // the prime
    uint64_t mu;     // floor(2^(63+k) / q)
    uint32_t shift;  // k - 1, k = bit length of q
    uint32_t pad;
    uint64_t n_inv;        // N^-1 mod q
    uint64_t n_inv_shoup;  // Shoup companion of n_inv
};

__device__ __forceinline__ uint64_t mulhi64(uint64_t a, uint64_t b) { return __umul64hi(a, b); }

__device__ __forceinline__ uint64_t csub(uint64_t x, uint64_t q) { return x >= q ? x - q : x; }

__device__ __forceinline__ uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) { return csub(a + b, q); }

__device__ __forceinline__ uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) { return a >= b ? a - b : a + q - b; }

// a * w mod q in [0, 2q), any a < 2^64
__device__ __forceinline__ uint64_t shoup_lazy(uint64_t a, uint64_t w, uint64_t ws, uint64_t q) {
    return a * w - mulhi64(a, ws) * q;
}

__device__ __forceinline__ uint64_t shoup(uint64_t a, uint64_t w, uint64_t ws, uint64_t q) {
    return csub(shoup_lazy(a, w, ws, q), q);
}

// 128-bit accumulator
struct u128 {
    uint64_t lo, hi;
};

__device__ __forceinline__ u128 mul_wide(uint64_t a, uint64_t b) { return {a * b, mulhi64(a, b)}; }

__device__ __forceinline__ void mac(u128 &acc, uint64_t a, uint64_t b) {
    uint64_t lo = a * b, hi = mulhi64(a, b);
    asm("add.cc.u64 %0, %0, %2;\n\taddc.u64 %1, %1, %3;" : "+l"(acc.lo), "+l"(acc.hi) : "l"(lo), "l"(hi));
}

__device__ __forceinline__ uint64_t barrett(u128 x, const PrimeConst &p) {
    uint64_t t = (x.hi << (64 - p.shift)) | (x.lo >> p.shift);
    uint64_t qh = mulhi64(t, p.mu);
    uint64_t r = x.lo - qh * p.q;
    r = csub(r, 2 * p.q);
    return csub(r, p.q);
}

__device__ __forceinline__ uint64_t mul_mod(uint64_t a, uint64_t b, const PrimeConst &p) {
    return barrett(mul_wide(a, b), p);
}

}  // namespace shm
