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
    uint32_t red_m;  // floor(2^(32+s) / q), s = max(0, k - 25): the multiplier of reduce_small
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

// a * w mod q in [0, 4q), any a < 2^64, with three 32-bit multiplies for the quotient
// instead of a full 64 x 64 high product.  With a = a1 2^32 + a0 and w' = s1 2^32 + s0,
// floor(a w' / 2^64) = a1 s1 + hi(a1 s0) + hi(a0 s1) + floor(F), where F collects the low
// words of the two cross products and a0 s0 / 2^64, so F < 3: dropping it leaves the
// quotient low by at most 2 and adds at most 2q to Shoup's remainder (below 2q).
__device__ __forceinline__ uint64_t shoup_lazy4(uint64_t a, uint64_t w, uint64_t ws, uint64_t q) {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
    const uint32_t s0 = (uint32_t)ws, s1 = (uint32_t)(ws >> 32);
    const uint64_t qh = (uint64_t)a1 * s1 + ((uint64_t)__umulhi(a1, s0) + __umulhi(a0, s1));
    return a * w - qh * q;
}

// x mod q for x < 2^(k+7), k = bit length of q.  With X = x >> s < 2^32 (s = max(0, k - 25))
// and red_m = floor(2^(32+s) / q) <= 2^8 (or < 2^32 when s = 0), qq = floor(X red_m / 2^32)
// never exceeds floor(x / q) and falls short of it by at most 2 (the truncations of X and
// of red_m each cost less than one, x_lo / q < 2^-24), so x - qq q lies in [0, 3q).
__device__ __forceinline__ uint64_t reduce_small(uint64_t x, const PrimeConst &p) {
    const uint32_t s = p.shift > 24 ? p.shift - 24 : 0;
    const uint32_t qq = __umulhi((uint32_t)(x >> s), p.red_m);
    uint64_t r = x - (uint64_t)qq * p.q;
    r = csub(r, 2 * p.q);
    return csub(r, p.q);
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

// Sum of products, generic (Acc<false>: 128-bit accumulator, any 64-bit operands) or for
// operands below 2^52 (Acc<true>, the limbs of primes below 2^52).  With a = a1 2^32 + a0
// and b = b1 2^32 + b0 (a1, b1 < 2^20), Acc<true> adds the 32 x 32-bit partial products into
// three 64-bit sums, hi = sum a1 b1, mid = sum (a0 b1 + a1 b0 + hi32(a0 b0)) and
// lo = sum lo32(a0 b0), which cannot overflow below 2^11 terms: four wide multiplies and no
// carry chain per term, one fold at the end.
template <bool S52>
struct Acc {
    u128 v{0, 0};
    __device__ __forceinline__ void add(uint64_t a, uint64_t b) { mac(v, a, b); }
    __device__ __forceinline__ u128 get() const { return v; }
};

template <>
struct Acc<true> {
    uint64_t lo = 0, mid = 0, hi = 0;
    __device__ __forceinline__ void add(uint64_t a, uint64_t b) {
        const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
        const uint64_t t = (uint64_t)a0 * b0;
        lo += (uint32_t)t;
        mid += (t >> 32) + (uint64_t)a0 * b1 + (uint64_t)a1 * b0;
        hi += (uint64_t)a1 * b1;
    }
    __device__ __forceinline__ u128 get() const {
        u128 x;
        x.lo = lo + (mid << 32);
        x.hi = hi + (mid >> 32) + (x.lo < lo ? 1 : 0);
        return x;
    }
};

// every prime of the chain below 2^52: the kernels may use Acc<true>
constexpr uint64_t kS52PrimeLimit = 1ull << 52;

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
