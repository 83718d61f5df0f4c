// Binary records of ciphertext batches, secrets and evaluation keys, so that
// keys and data move between processes and can be imported for parity runs.
//
// The reference keeps its objects in device memory and reads one thing from a file: a
// secret key as decimal NTT-form residues over every prime of the key level, one per line
// (PhantomSecretKey::load_secret_key, thirdparty/phantom-fhe/include/secretkey.h:290-307).
// import_secret_text reads that format and export_secret_text writes it; the NTT form and
// prime order are the reference's, so a secret moves either way unchanged.
//
// A record is an 80-byte header, the payload as little-endian 64-bit words, and the
// record's digest (8 bytes).  Header, in order:
//   magic "SHMOAIW\0" (8 bytes), version (u16, 1), kind (u16, Kind),
//   log N (u32), n_q (u32), n_p (u32), digest of the prime chain Q then P (u64),
//   shape d0, d1, d2 (u32 each), flags (u32: bit 0 shared-a groups),
//   tag (u32: Galois element or member index), group (u32: members of a shared-a key set,
//   or the number of auxiliary secrets), scale (f64), payload words (u64), reserved (u64, 0).
// The payload holds d0 * d1 * d2 * N words.  The digest covers the header (its 80 bytes as
// ten little-endian words) and then the payload: 64-bit FNV-1a over words,
// h = (h ^ w) * 0x100000001b3, starting from 0xcbf29ce484222325.
//
// Loading checks every header field against the context, every residue against its prime
// (every secret coefficient against |c| < 2^31) and the digest, and throws Error (code
// SHM_EINVAL) before anything is returned when one fails.
#pragma once

#include <cstdint>
#include <functional>
#include <iosfwd>
#include <map>
#include <vector>

#include "host.hpp"

namespace shmoai {
namespace wire {

enum class Kind : uint16_t {
    Ciphertext = 1,       // d0 = count, d1 = size, d2 = L; flags bit 0 for shared-a groups
                          // (2 is not assigned)
    Secret = 3,           // d0 = 1 + auxiliary secrets, d1 = d2 = 1; signed coefficients
    RelinKey = 4,         // d0 = dnum, d1 = 2, d2 = QP
    GaloisKey = 5,        // the same, tag = Galois element
    SharedGaloisKey = 6,  // d0 = dnum, d1 = members + 1, d2 = QP; tag = element, group = members
    FormatKey = 7,        // d0 = members, d1 = members + 1, d2 = QP; group = members
    BackwardKey = 8,      // d0 = dnum, d1 = 2, d2 = QP; tag = member, group = members
    End = 9,              // closes a key stream; no payload words
};

using Sink = std::function<void(const void *, size_t)>;
using Source = std::function<void(void *, size_t)>;  // must fill all bytes or throw

constexpr size_t kHeaderBytes = 80;

// one ciphertext batch
size_t serialized_bytes(const Context &c, const Ciphertext &ct);
void save(const Sink &out, const Context &c, const Ciphertext &ct);
Ciphertext load_ciphertext(const Source &in, const Context &c);

// A key stream: the secrets (optional), the relinearisation key, Galois keys, and the
// shared-a key sets, then an End record.  Missing pointers are skipped.
struct KeySet {
    const std::vector<int64_t> *secret = nullptr;
    const std::vector<std::vector<int64_t>> *aux = nullptr;
    const DeviceBuffer *relin = nullptr;
    const std::map<uint32_t, DeviceBuffer> *galois = nullptr;
    const std::map<uint32_t, SharedAKeys> *shared = nullptr;
};
void save_keys(const Sink &out, const Context &c, const KeySet &keys);

struct LoadedKeys {
    bool has_secret = false;
    std::vector<int64_t> secret;
    std::vector<std::vector<int64_t>> aux;
    DeviceBuffer relin;  // empty when the stream has none
    std::map<uint32_t, DeviceBuffer> galois;
    std::map<uint32_t, SharedAKeys> shared;  // complete sets only (format + every backward key)
};
LoadedKeys load_keys(const Source &in, const Context &c);

// the reference's secret-key text: Q·P·N decimal residues, limb-major, NTT form
std::vector<int64_t> import_secret_text(std::istream &in, const Context &c);
void export_secret_text(std::ostream &out, const Context &c, const std::vector<int64_t> &secret);

// digest of the prime chain, as the header carries it
uint64_t chain_digest(const Context &c);

}  // namespace wire
}  // namespace shmoai
