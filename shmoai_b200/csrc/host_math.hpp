// Host-side number theory for the CKKS context: prime chain, NTT twiddle
// tables, Shoup/Barrett constants and RNS base-conversion constants.
//
// The prime chain and twiddle order follow the reference so that limbs are
// bit-identical: CoeffModulus::Create (thirdparty/phantom-fhe/src/modulus.cu:79-110)
// searches primes = 1 mod 2N downwards from 2^b - 2N + 1 (src/util/numth.cu:209-235)
// and hands each request of a bit size the last remaining prime of that size;
// the NTT uses the smallest primitive 2N-th root psi with
// root_powers[bitrev(i)] = psi^i (src/util/ntt.cu:11-56).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <vector>

namespace shm::host {

using u128 = unsigned __int128;

inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)((u128)a * b % q); }

inline uint64_t powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    for (; e; e >>= 1) {
        if (e & 1) r = mulmod(r, a, q);
        a = mulmod(a, a, q);
    }
    return r;
}

inline uint64_t invmod(uint64_t a, uint64_t q) { return powmod(a % q, q - 2, q); }

inline int bit_length(uint64_t x) { return 64 - __builtin_clzll(x); }

inline bool is_prime(uint64_t n) {
    if (n < 2) return false;
    for (uint64_t p : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
        if (n % p == 0) return n == p;
    }
    uint64_t d = n - 1;
    int s = 0;
    while (!(d & 1)) d >>= 1, s++;
    for (uint64_t a : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
        uint64_t x = powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool witness = true;
        for (int r = 1; r < s && witness; r++) {
            x = mulmod(x, x, n);
            if (x == n - 1) witness = false;
        }
        if (witness) return false;
    }
    return true;
}

// Prime chain for the requested bit sizes (see the header comment for the order).
inline std::vector<uint64_t> create_primes(int log_n, const std::vector<int> &bits) {
    const uint64_t step = 2ull << log_n;
    std::vector<uint64_t> out(bits.size());
    for (size_t i = 0; i < bits.size(); i++) {
        int b = bits[i];
        if (b < 20 || b > 61) throw std::invalid_argument("prime bit size must be in [20, 61]");
        size_t total = 0, earlier = 0;
        for (size_t k = 0; k < bits.size(); k++) {
            if (bits[k] != b) continue;
            total++;
            if (k < i) earlier++;
        }
        size_t want = total - 1 - earlier, found = 0;
        uint64_t v = (1ull << b) - step + 1, lower = 1ull << (b - 1);
        bool got = false;
        for (; v > lower; v -= step) {
            if (!is_prime(v)) continue;
            if (found++ == want) {
                out[i] = v;
                got = true;
                break;
            }
        }
        if (!got) throw std::invalid_argument("not enough NTT-friendly primes of the requested size");
    }
    return out;
}

inline uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; i++, x >>= 1) r = (r << 1) | (x & 1);
    return r;
}

inline uint64_t minimal_root(uint64_t q, int log_n) {
    const uint64_t two_n = 2ull << log_n, n = 1ull << log_n;
    if ((q - 1) % two_n) throw std::invalid_argument("prime is not 1 mod 2N");
    uint64_t g = 0;
    for (uint64_t x = 2;; x++) {
        uint64_t r = powmod(x, (q - 1) / two_n, q);
        if (powmod(r, n, q) == q - 1) {
            g = r;
            break;
        }
    }
    uint64_t sq = mulmod(g, g, q), cur = g, best = g;
    for (uint64_t i = 0; i < n; i++) {
        if (cur < best) best = cur;
        cur = mulmod(cur, sq, q);
    }
    return best;
}

inline uint64_t shoup_of(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }

inline uint64_t barrett_mu(uint64_t q) {
    int k = bit_length(q);
    return (uint64_t)(((u128)1 << (63 + k)) / q);
}

// psi^i at bitrev(i) and psi^-i at bitrev(i), with Shoup companions
inline void ntt_tables(uint64_t q, int log_n, uint64_t *rp, uint64_t *rps, uint64_t *irp, uint64_t *irps) {
    const uint32_t n = 1u << log_n;
    uint64_t psi = minimal_root(q, log_n), ipsi = invmod(psi, q), p = 1, ip = 1;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t r = bitrev(i, log_n);
        rp[r] = p;
        rps[r] = shoup_of(p, q);
        irp[r] = ip;
        irps[r] = shoup_of(ip, q);
        p = mulmod(p, psi, q);
        ip = mulmod(ip, ipsi, q);
    }
}

// prod_{k in set, k != i} m_k  mod t
inline uint64_t partial_product(const std::vector<uint64_t> &mods, size_t skip, uint64_t t) {
    uint64_t h = 1 % t;
    for (size_t k = 0; k < mods.size(); k++)
        if (k != skip) h = mulmod(h, mods[k] % t, t);
    return h;
}

}  // namespace shm::host
