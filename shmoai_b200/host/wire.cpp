// Binary records of ciphertexts, secrets and keys (include/shmoai/wire.hpp).
#include "../../include/shmoai/wire.hpp"

#include <cstring>
#include <istream>
#include <ostream>
#include <string>

#include "internal.hpp"

static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "records are little-endian words");

namespace shmoai {
namespace wire {
namespace {

constexpr char kMagic[8] = {'S', 'H', 'M', 'O', 'A', 'I', 'W', '\0'};
constexpr uint16_t kVersion = 1;
constexpr uint64_t kFnvBasis = 0xcbf29ce484222325ull, kFnvPrime = 0x100000001b3ull;
constexpr int64_t kSecretLimit = int64_t(1) << 31;
constexpr uint32_t kFlagShared = 1;
constexpr size_t kChunkWords = size_t(1) << 22;  // 32 MB per host staging chunk

uint64_t fnv(uint64_t h, const uint64_t *w, size_t n) {
    for (size_t i = 0; i < n; i++) h = (h ^ w[i]) * kFnvPrime;
    return h;
}

struct Header {
    Kind kind = Kind::End;
    uint32_t log_n = 0, nq = 0, np = 0;
    uint64_t chain = 0;
    uint32_t d0 = 0, d1 = 0, d2 = 0, flags = 0, tag = 0, group = 0;
    double scale = 1.0;
    uint64_t words = 0;
    uint64_t digest = 0;  // of the header's bytes: the record's digest continues from it
};

uint64_t header_digest(const uint8_t *b) {
    uint64_t w[kHeaderBytes / 8];
    std::memcpy(w, b, kHeaderBytes);
    return fnv(kFnvBasis, w, kHeaderBytes / 8);
}

template <typename T>
void put(uint8_t *&p, T v) {
    std::memcpy(p, &v, sizeof v);
    p += sizeof v;
}
template <typename T>
T get(const uint8_t *&p) {
    T v;
    std::memcpy(&v, p, sizeof v);
    p += sizeof v;
    return v;
}

uint64_t write_header(const Sink &out, const Header &h) {
    uint8_t b[kHeaderBytes] = {}, *p = b;
    std::memcpy(p, kMagic, 8);
    p += 8;
    put<uint16_t>(p, kVersion);
    put<uint16_t>(p, (uint16_t)h.kind);
    put(p, h.log_n);
    put(p, h.nq);
    put(p, h.np);
    put(p, h.chain);
    put(p, h.d0);
    put(p, h.d1);
    put(p, h.d2);
    put(p, h.flags);
    put(p, h.tag);
    put(p, h.group);
    put(p, h.scale);
    put(p, h.words);
    put<uint64_t>(p, 0);  // reserved
    out(b, kHeaderBytes);
    return header_digest(b);
}

Header read_header(const Source &in, const Context &c) {
    uint8_t b[kHeaderBytes];
    in(b, kHeaderBytes);
    if (std::memcmp(b, kMagic, 8) != 0) throw Error("not a record: bad magic");
    const uint8_t *p = b + 8;
    Header h;
    h.digest = header_digest(b);
    const uint16_t version = get<uint16_t>(p);
    if (version != kVersion) throw Error("record version " + std::to_string(version) + " is not supported");
    const uint16_t kind = get<uint16_t>(p);
    if (kind < (uint16_t)Kind::Ciphertext || kind > (uint16_t)Kind::End)
        throw Error("unknown record kind " + std::to_string(kind));
    h.kind = (Kind)kind;
    h.log_n = get<uint32_t>(p);
    h.nq = get<uint32_t>(p);
    h.np = get<uint32_t>(p);
    h.chain = get<uint64_t>(p);
    h.d0 = get<uint32_t>(p);
    h.d1 = get<uint32_t>(p);
    h.d2 = get<uint32_t>(p);
    h.flags = get<uint32_t>(p);
    h.tag = get<uint32_t>(p);
    h.group = get<uint32_t>(p);
    h.scale = get<double>(p);
    h.words = get<uint64_t>(p);
    if (get<uint64_t>(p) != 0) throw Error("reserved header field is not zero");
    if (h.log_n != c.log_n || h.nq != c.nq || h.np != c.np || h.chain != chain_digest(c))
        throw Error("record was written for another ring or prime chain");
    if ((unsigned __int128)h.d0 * h.d1 * h.d2 * c.n != h.words) throw Error("record shape and word count disagree");
    return h;
}

Header base(const Context &c, Kind k) {
    Header h;
    h.kind = k;
    h.log_n = c.log_n;
    h.nq = c.nq;
    h.np = c.np;
    h.chain = chain_digest(c);
    return h;
}

// device words -> sink, in chunks, then the digest (continued from the header's)
void write_device(const Sink &out, const Context &c, const uint64_t *dev, size_t words, uint64_t h) {
    std::vector<uint64_t> buf(std::min(words, kChunkWords));
    for (size_t off = 0; off < words; off += buf.size()) {
        const size_t n = std::min(buf.size(), words - off);
        c.check(shm_memcpy(c.handle(), buf.data(), dev + off, n * 8, SHM_COPY_D2H, c.stream()));
        h = fnv(h, buf.data(), n);
        out(buf.data(), n * 8);
    }
    out(&h, 8);
}

// source -> device words, in chunks; limb j of every [d2][N] block must be below primes[j]
void read_device(const Source &in, const Context &c, uint64_t *dev, size_t words,
                 const std::vector<uint64_t> &limb_primes, uint64_t h) {
    const size_t N = c.n, d2 = limb_primes.size();
    std::vector<uint64_t> buf(std::min(words, (kChunkWords / N) * N));
    for (size_t off = 0; off < words; off += buf.size()) {
        const size_t n = std::min(buf.size(), words - off);
        in(buf.data(), n * 8);
        h = fnv(h, buf.data(), n);
        for (size_t r = 0; r < n / N; r++) {
            const size_t row = off / N + r;
            const uint64_t q = limb_primes[row % d2], *w = buf.data() + r * N;
            for (size_t k = 0; k < N; k++)
                if (w[k] >= q)
                    throw Error("residue " + std::to_string(w[k]) + " at row " + std::to_string(row) +
                                " is not below its prime " + std::to_string(q));
        }
        c.check(shm_memcpy(c.handle(), dev + off, buf.data(), n * 8, SHM_COPY_H2D, c.stream()));
    }
    uint64_t stored;
    in(&stored, 8);
    if (stored != h) throw Error("digest mismatch: the record is corrupt");
}

std::vector<uint64_t> q_primes(const Context &c, uint32_t L) {
    return std::vector<uint64_t>(c.primes.begin(), c.primes.begin() + L);
}
std::vector<uint64_t> qp_primes(const Context &c) { return c.primes; }

Header expect(const Source &in, const Context &c, Kind k) {
    Header h = read_header(in, c);
    if (h.kind != k)
        throw Error("record kind " + std::to_string((int)h.kind) + " where " + std::to_string((int)k) +
                    " was expected");
    return h;
}

void key_record(const Sink &out, const Context &c, Kind k, const DeviceBuffer &key, uint32_t d0, uint32_t d1,
                uint32_t tag, uint32_t group) {
    const uint32_t QP = c.nq + c.np;
    if (key.words() != (size_t)d0 * d1 * QP * c.n) throw Error("key buffer has the wrong size for its kind");
    Header h = base(c, k);
    h.d0 = d0;
    h.d1 = d1;
    h.d2 = QP;
    h.tag = tag;
    h.group = group;
    h.words = key.words();
    write_device(out, c, key.data(), key.words(), write_header(out, h));
}

DeviceBuffer key_payload(const Source &in, const Context &c, const Header &h, uint32_t d0, uint32_t d1) {
    if (h.d0 != d0 || h.d1 != d1 || h.d2 != c.nq + c.np) throw Error("key record has the wrong shape");
    DeviceBuffer key(c, h.words);
    read_device(in, c, key.data(), h.words, qp_primes(c), h.digest);
    return key;
}

std::vector<int64_t> check_secret(std::vector<int64_t> s, const Context &c) {
    if (s.size() != c.n) throw Error("secret has the wrong length");
    for (int64_t v : s)
        if (v <= -kSecretLimit || v >= kSecretLimit) throw Error("secret coefficient out of range");
    return s;
}

}  // namespace

uint64_t chain_digest(const Context &c) { return fnv(kFnvBasis, c.primes.data(), c.primes.size()); }

size_t serialized_bytes(const Context &c, const Ciphertext &ct) {
    return kHeaderBytes + ct.polys() * ct.L * c.n * 8 + 8;
}

void save(const Sink &out, const Context &c, const Ciphertext &ct) {
    Header h = base(c, Kind::Ciphertext);
    h.d0 = ct.count;
    h.d1 = ct.size;
    h.d2 = ct.L;
    h.flags = ct.shared ? kFlagShared : 0;
    h.scale = ct.scale_;
    h.words = ct.polys() * ct.L * c.n;
    if (ct.data.words() < h.words) throw Error("ciphertext buffer smaller than its shape");
    write_device(out, c, ct.data.data(), h.words, write_header(out, h));
}

Ciphertext load_ciphertext(const Source &in, const Context &c) {
    const Header h = expect(in, c, Kind::Ciphertext);
    if (!h.d0 || !h.d1 || !h.d2 || h.d2 > c.nq) throw Error("ciphertext record has an invalid shape");
    if (h.flags & ~kFlagShared) throw Error("ciphertext record has unknown flags");
    if ((h.flags & kFlagShared) && h.d1 < 2) throw Error("shared-a group without members");
    if (!(h.flags & kFlagShared) && h.d1 > 3) throw Error("ciphertext size above 3");
    Ciphertext ct;
    ct.data = DeviceBuffer(c, h.words);
    read_device(in, c, ct.data.data(), h.words, q_primes(c, h.d2), h.digest);
    ct.count = h.d0;
    ct.size = h.d1;
    ct.L = h.d2;
    ct.scale_ = h.scale;
    ct.shared = (h.flags & kFlagShared) != 0;
    return ct;
}

void save_keys(const Sink &out, const Context &c, const KeySet &keys) {
    if (keys.secret) {
        std::vector<const std::vector<int64_t> *> rows{keys.secret};
        if (keys.aux)
            for (auto &a : *keys.aux) rows.push_back(&a);
        Header h = base(c, Kind::Secret);
        h.d0 = (uint32_t)rows.size();
        h.d1 = h.d2 = 1;
        h.group = (uint32_t)rows.size() - 1;
        h.words = rows.size() * c.n;
        uint64_t d = write_header(out, h);
        for (auto *r : rows) {
            if (r->size() != c.n) throw Error("secret has the wrong length");
            d = fnv(d, reinterpret_cast<const uint64_t *>(r->data()), c.n);
            out(r->data(), c.n * 8);
        }
        out(&d, 8);
    }
    if (keys.relin && keys.relin->data()) key_record(out, c, Kind::RelinKey, *keys.relin, c.dnum, 2, 0, 0);
    if (keys.galois)
        for (auto &kv : *keys.galois) key_record(out, c, Kind::GaloisKey, kv.second, c.dnum, 2, kv.first, 0);
    if (keys.shared)
        for (auto &kv : *keys.shared) {
            const SharedAKeys &s = kv.second;
            const uint32_t m = s.members;
            if (s.backward.size() != m) throw Error("shared-a key set without its backward keys");
            key_record(out, c, Kind::FormatKey, s.format, m, m + 1, 0, m);
            for (uint32_t i = 0; i < m; i++) key_record(out, c, Kind::BackwardKey, s.backward[i], c.dnum, 2, i, m);
            for (auto &g : s.galois) key_record(out, c, Kind::SharedGaloisKey, g.second, c.dnum, m + 1, g.first, m);
        }
    Header end = base(c, Kind::End);
    const uint64_t d = write_header(out, end);
    out(&d, 8);
}

LoadedKeys load_keys(const Source &in, const Context &c) {
    LoadedKeys k;
    std::map<uint32_t, std::vector<bool>> have_backward;
    std::map<uint32_t, bool> have_format;
    for (;;) {
        const Header h = read_header(in, c);
        switch (h.kind) {
            case Kind::End: {
                uint64_t d;
                in(&d, 8);
                if (d != h.digest || h.words) throw Error("malformed end record");
                for (auto &kv : k.shared) {
                    bool complete = have_format[kv.first];
                    for (bool b : have_backward[kv.first]) complete = complete && b;
                    if (!complete)
                        throw Error("shared-a key set of " + std::to_string(kv.first) + " members is incomplete");
                }
                return k;
            }
            case Kind::Secret: {
                if (h.d0 < 1 || h.d0 > 257 || h.d1 != 1 || h.d2 != 1 || h.group != h.d0 - 1)
                    throw Error("secret record has an invalid shape");
                std::vector<uint64_t> w(h.words);
                in(w.data(), h.words * 8);
                uint64_t d;
                in(&d, 8);
                if (d != fnv(h.digest, w.data(), w.size())) throw Error("digest mismatch: the record is corrupt");
                auto row = [&](uint32_t r) {
                    std::vector<int64_t> s(c.n);
                    std::memcpy(s.data(), w.data() + (size_t)r * c.n, c.n * 8);
                    return check_secret(std::move(s), c);
                };
                k.has_secret = true;
                k.secret = row(0);
                k.aux.clear();
                for (uint32_t r = 1; r < h.d0; r++) k.aux.push_back(row(r));
                break;
            }
            case Kind::RelinKey:
                k.relin = key_payload(in, c, h, c.dnum, 2);
                break;
            case Kind::GaloisKey:
                k.galois[h.tag] = key_payload(in, c, h, c.dnum, 2);
                break;
            case Kind::FormatKey:
            case Kind::BackwardKey:
            case Kind::SharedGaloisKey: {
                const uint32_t m = h.group;
                if (!m) throw Error("shared-a key record without a group size");
                SharedAKeys &s = k.shared[m];
                s.members = m;
                if (s.backward.size() != m) s.backward.resize(m);
                have_backward[m].resize(m, false);
                if (h.kind == Kind::FormatKey) {
                    s.format = key_payload(in, c, h, m, m + 1);
                    have_format[m] = true;
                } else if (h.kind == Kind::BackwardKey) {
                    if (h.tag >= m) throw Error("backward key of a member outside the group");
                    s.backward[h.tag] = key_payload(in, c, h, c.dnum, 2);
                    have_backward[m][h.tag] = true;
                } else {
                    s.galois[h.tag] = key_payload(in, c, h, c.dnum, m + 1);
                }
                break;
            }
            default:
                throw Error("record kind " + std::to_string((int)h.kind) + " does not belong in a key stream");
        }
    }
}

std::vector<int64_t> import_secret_text(std::istream &in, const Context &c) {
    const uint32_t QP = c.nq + c.np;
    const size_t words = (size_t)QP * c.n;
    std::vector<uint64_t> w;
    w.reserve(words);
    std::string line;
    while (std::getline(in, line)) {
        size_t a = line.find_first_not_of(" \t\r");
        if (a == std::string::npos) continue;
        size_t used = 0;
        uint64_t v;
        try {
            v = std::stoull(line.substr(a), &used);
        } catch (const std::exception &) {
            throw Error("secret text: line " + std::to_string(w.size() + 1) + " is not a number");
        }
        if (line.find_first_not_of(" \t\r", a + used) != std::string::npos)
            throw Error("secret text: trailing characters on line " + std::to_string(w.size() + 1));
        if (w.size() == words) throw Error("secret text holds more than Q*P*N residues");
        if (v >= c.primes[w.size() / c.n]) throw Error("secret text: residue not below its prime");
        w.push_back(v);
    }
    if (w.size() != words) throw Error("secret text holds " + std::to_string(w.size()) + " residues, expected " +
                                       std::to_string(words));
    DeviceBuffer d(c, words);
    c.check(shm_memcpy(c.handle(), d.data(), w.data(), words * 8, SHM_COPY_H2D, c.stream()));
    c.check(shm_ntt_inverse(c.handle(), d.data(), 1, QP, c.stream()));
    c.check(shm_memcpy(c.handle(), w.data(), d.data(), words * 8, SHM_COPY_D2H, c.stream()));
    // the coefficients are small integers: centre limb 0, then every other limb must agree
    std::vector<int64_t> s(c.n);
    const uint64_t q0 = c.primes[0];
    for (size_t k = 0; k < c.n; k++) s[k] = w[k] > q0 / 2 ? -(int64_t)(q0 - w[k]) : (int64_t)w[k];
    for (uint32_t j = 1; j < QP; j++) {
        const uint64_t q = c.primes[j];
        for (size_t k = 0; k < c.n; k++) {
            const uint64_t want = s[k] < 0 ? q - (uint64_t)(-s[k]) % q : (uint64_t)s[k] % q;
            if (w[(size_t)j * c.n + k] != (want == q ? 0 : want))
                throw Error("secret text: the limbs do not hold one small integer polynomial");
        }
    }
    return check_secret(std::move(s), c);
}

void export_secret_text(std::ostream &out, const Context &c, const std::vector<int64_t> &secret) {
    const uint32_t QP = c.nq + c.np;
    const size_t words = (size_t)QP * c.n;
    check_secret(secret, c);
    DeviceBuffer d(c, words);
    Encoder(c).upload(secret.data(), 1, QP, d.data());
    std::vector<uint64_t> w(words);
    c.check(shm_memcpy(c.handle(), w.data(), d.data(), words * 8, SHM_COPY_D2H, c.stream()));
    for (uint64_t v : w) out << v << '\n';
    if (!out) throw Error("secret text: write failed");
}

}  // namespace wire
}  // namespace shmoai
