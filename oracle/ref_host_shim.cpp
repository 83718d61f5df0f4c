// Thin extern "C" face over the reference's own host-side number theory
// (ShMOAI's vendored PhantomFHE: src/modulus.cu, src/util/ntt.cu,
// src/util/numth.cu, src/util/rns.cu), compiled from the reference sources by
// oracle/build_ref.sh into oracle/_ref/libref_host.so.
//
// TEST INFRASTRUCTURE ONLY: the tests use it to pin the oracle's prime chain,
// NTT tables and RNS base-conversion constants to the reference's.
#include <cstdint>
#include <cstring>
#include <vector>

#include "util/modulus.h"
#include "util/ntt.h"
#include "util/rns.h"

using namespace phantom::arith;

extern "C" {

// CoeffModulus::Create(2^log_n, bits) -> primes (modulus.cu:79-110).
int ref_create_primes(uint32_t log_n, const int *bits, uint32_t count, uint64_t *out) {
    try {
        std::vector<int> b(bits, bits + count);
        auto mods = CoeffModulus::Create(size_t(1) << log_n, b);
        for (uint32_t i = 0; i < count; i++) out[i] = mods[i].value();
        return 0;
    } catch (...) {
        return -1;
    }
}

// NTT tables of one prime (util/ntt.cu:11-56): forward root powers, inverse
// root powers (with N^-1 folded into entry 1, as the reference stores them),
// the root itself and N^-1 mod q.
int ref_ntt_tables(uint32_t log_n, uint64_t q, uint64_t *rp, uint64_t *irp, uint64_t *root, uint64_t *n_inv) {
    try {
        NTT t((int)log_n, Modulus(q));
        size_t n = size_t(1) << log_n;
        std::memcpy(rp, t.get_from_root_powers().data(), n * sizeof(uint64_t));
        std::memcpy(irp, t.get_from_inv_root_powers().data(), n * sizeof(uint64_t));
        *root = t.get_root();
        *n_inv = t.inv_degree_modulo();
        return 0;
    } catch (...) {
        return -1;
    }
}

// Base conversion constants ibase -> obase (util/rns.cu, BaseConverter):
// qhat_inv[i] = (Q/q_i)^-1 mod q_i and qhat_mod_p[j * n_in + i] = (Q/q_i) mod p_j.
int ref_base_converter(const uint64_t *ibase, uint32_t n_in, const uint64_t *obase, uint32_t n_out,
                       uint64_t *qhat_inv, uint64_t *qhat_mod_p) {
    try {
        std::vector<Modulus> im, om;
        for (uint32_t i = 0; i < n_in; i++) im.emplace_back(ibase[i]);
        for (uint32_t j = 0; j < n_out; j++) om.emplace_back(obase[j]);
        RNSBase ib(im), ob(om);
        BaseConverter conv(ib, ob);
        std::memcpy(qhat_inv, ib.QHatInvModq(), n_in * sizeof(uint64_t));
        for (uint32_t j = 0; j < n_out; j++) std::memcpy(qhat_mod_p + (size_t)j * n_in, conv.QHatModp(j), n_in * sizeof(uint64_t));
        return 0;
    } catch (...) {
        return -1;
    }
}
}
