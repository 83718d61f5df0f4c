// Internal helpers of the C++ host library.
#pragma once

#include <cstdint>

#include "../../include/shmoai/host.hpp"

namespace shmoai {
namespace detail {

using u128 = unsigned __int128;

inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }
inline uint64_t addmod(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t s = a + b;
    return s >= q ? s - q : s;
}
inline uint64_t powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = mulmod(r, a, q);
        a = mulmod(a, a, q);
        e >>= 1;
    }
    return r;
}

// splitmix64 output mix of seed + (idx + 1) * golden gamma; the device samplers use the
// same function, so host-drawn and device-drawn values agree
inline uint64_t mix64(uint64_t seed, uint64_t idx) {
    uint64_t z = seed + (idx + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Chebyshev series on ciphertexts (chebyshev.cpp): the basis T_1 .. T_8, T_16, T_32, .. up
// to `deg`, whether a series of ncoef coefficients fits from level lvl, and its baby-step
// giant-step evaluation at scale S and lvl primes
using ChebBasis = std::map<int, Ciphertext>;
void cheb_divide(const std::vector<double> &c, int m, std::vector<double> &q, std::vector<double> &r);
int bitlen(uint32_t d);
ChebBasis cheb_basis(const Evaluator &ev, const Ciphertext &x, int deg);
bool cheb_feasible(const ChebBasis &T, int ncoef, uint32_t lvl);
Ciphertext cheb_eval(const Evaluator &ev, const ChebBasis &T, const std::vector<double> &c, double S, uint32_t lvl,
                     bool lazy = false);

}  // namespace detail
}  // namespace shmoai
