"""Binary records of ciphertexts and keys (include/shmoai/wire.hpp, shm_ct_serialize /
shm_host_save_keys / shm_host_load_keys) and the reference's secret-key text
(PhantomSecretKey::load_secret_key, thirdparty/phantom-fhe/include/secretkey.h:290-307:
NTT-form residues over every prime of the key level, one decimal per line).

CPU: the host library on the oracle's C ABI.  Round trips are bit-exact; a record is parsed
here from the documented layout (so the layout itself is pinned); every kind of damage
(digest, truncation, trailing bytes, another prime chain, a residue at or above its prime,
bad magic) is refused with a message; keys moved to a second host with another seed give
bit-identical evaluator results; a secret written here in the reference's text format from
the oracle's NTT (pinned to the reference's twiddles) decrypts the same ciphertexts, and
exporting it gives the same text back.  GPU: records written by the CUDA build and by the
oracle build are the same bytes and load in the other build.
"""
import ctypes
import os
import struct

import numpy as np
import pytest

from oracle import oracle as O
from shmoai_b200.host import Host, HostError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_HOST = os.path.join(ROOT, "oracle", "_build", "libshmoai_host_oracle.so")
LOG_N = 12
BITS = [51, 46, 46, 46, 46, 51] + [51, 51]  # N = 2^12, nq = 6, np = 2 (dnum 3)
NP = 2
HEADER = struct.Struct("<8sHHIIIQIIIIIIdQQ")
FNV_BASIS, FNV_PRIME = 0xCBF29CE484222325, 0x100000001B3
M64 = (1 << 64) - 1


def _primes():
    return [int(p) for p in O.gen_primes(LOG_N, BITS)]


def _host(seed=11, lib=ORACLE_HOST, primes=None):
    return Host(LOG_N, primes or _primes(), NP, hamming_weight=64, seed=seed, lib=lib)


def _z(rng, count, n):
    return rng.uniform(-1, 1, (count, n)) + 1j * rng.uniform(-1, 1, (count, n))


def _fnv(words):
    h = FNV_BASIS
    for w in np.asarray(words, dtype=np.uint64).tolist():
        h = ((h ^ w) * FNV_PRIME) & M64
    return h


def _records(blob):
    """Split a byte string of records into (header fields, payload words, digest)."""
    out, off = [], 0
    while off < len(blob):
        f = HEADER.unpack_from(blob, off)
        words = f[-2]
        assert f[-1] == 0
        off += HEADER.size
        payload = np.frombuffer(blob, dtype=np.uint64, count=words, offset=off)
        off += 8 * words
        digest = struct.unpack_from("<Q", blob, off)[0]
        off += 8
        out.append((f, payload, digest))
    return out


def test_header_layout_is_80_bytes():
    assert HEADER.size == 80


def test_ciphertext_record_round_trip_and_layout():
    h = _host()
    rng = np.random.default_rng(1)
    ct = h.encrypt(_z(rng, 2, 64), 2.0 ** 40, 4)
    blob = ct.serialize()
    (f, payload, digest), = _records(blob)
    magic, ver, kind, log_n, nq, np_, chain, d0, d1, d2, flags, tag, group, scale, words, _ = f
    assert (magic, ver, kind, log_n, nq, np_) == (b"SHMOAIW\0", 1, 1, LOG_N, 6, NP)
    assert chain == _fnv(h.primes)
    assert (d0, d1, d2, flags, scale, words) == (2, 2, 4, 0, 2.0 ** 40, 2 * 2 * 4 * h.n)
    assert np.array_equal(payload.reshape(2, 2, 4, h.n), ct.to_host())
    assert digest == _fnv(np.concatenate([np.frombuffer(blob[:HEADER.size], dtype=np.uint64), payload]))
    back = h.deserialize(blob)
    assert (back.count, back.size, back.level, back.scale, back.shared) == (2, 2, 4, 2.0 ** 40, False)
    assert np.array_equal(back.to_host(), ct.to_host())
    # a shared-a batch keeps its flag
    h.gen_relin_key()
    h.gen_shared_keys(2, [h.galois_elt(1)], hamming_weight=64)
    sh = h.to_shared(h.encrypt(_z(rng, 4, 64), 2.0 ** 40, 3), 2)
    sb = sh.serialize()
    assert _records(sb)[0][0][10] == 1
    back = h.deserialize(sb)
    assert back.shared and back.members == 2 and np.array_equal(back.to_host(), sh.to_host())
    assert np.abs(h.decrypt(back) - h.decrypt(sh)).max() == 0


def _forge(blob, payload):
    """The record with `payload` in place of its own and the digest recomputed."""
    head = blob[:HEADER.size]
    words = np.concatenate([np.frombuffer(head, dtype=np.uint64), payload])
    return head + payload.tobytes() + struct.pack("<Q", _fnv(words))


def test_damaged_records_are_refused():
    h = _host()
    ct = h.encrypt(_z(np.random.default_rng(2), 1, 16), 2.0 ** 40, 3)
    blob = bytearray(ct.serialize())
    bad = bytearray(blob)
    bad[HEADER.size + 100] ^= 1
    with pytest.raises(HostError, match="digest"):
        h.deserialize(bytes(bad))
    with pytest.raises(HostError, match="truncated"):
        h.deserialize(bytes(blob[:-9]))
    for off in (48, 56, 63):  # tag, scale: fields no shape check reads are covered by the digest
        bad = bytearray(blob)
        bad[off] ^= 4
        with pytest.raises(HostError, match="digest"):
            h.deserialize(bytes(bad))
    with pytest.raises(HostError, match="bytes after"):
        h.deserialize(bytes(blob) + b"\0")
    bad = bytearray(blob)
    bad[0:1] = b"X"
    with pytest.raises(HostError, match="magic"):
        h.deserialize(bytes(bad))
    bad = bytearray(blob)
    struct.pack_into("<I", bad, 12, LOG_N + 1)
    with pytest.raises(HostError, match="another ring"):
        h.deserialize(bytes(bad))
    bad = bytearray(blob)
    struct.pack_into("<I", bad, 32 + 4, 5)  # d1 = 5 with the same word count
    with pytest.raises(HostError, match="disagree"):
        h.deserialize(bytes(bad))
    payload = np.frombuffer(bytes(blob), dtype=np.uint64, count=3 * 2 * h.n, offset=HEADER.size).copy()
    payload[h.n + 7] = h.primes[1]  # limb 1 of c0 holds q_1 itself
    with pytest.raises(HostError, match="not below its prime"):
        h.deserialize(_forge(bytes(blob), payload))
    other = _host(primes=[int(p) for p in O.gen_primes(LOG_N, [51, 46, 46, 46, 46, 50, 51, 51])])
    with pytest.raises(HostError, match="prime chain"):
        other.deserialize(bytes(blob))


def test_keys_move_to_another_host(tmp_path):
    a, b = _host(seed=11), _host(seed=99)
    rng = np.random.default_rng(3)
    a.gen_relin_key()
    elts = [a.galois_elt(1), a.galois_elt(-2)]
    a.gen_galois_keys(elts)
    a.gen_shared_keys(2, elts, hamming_weight=64)
    path = str(tmp_path / "keys.bin")
    a.save_keys(path)
    x, y = a.encrypt(_z(rng, 2, 64), 2.0 ** 40, 5), a.encrypt(_z(rng, 2, 64), 2.0 ** 40, 5)
    assert np.abs(b.decrypt(x) - a.decrypt(x)).max() > 1e-2  # another secret before loading
    b.load_keys(path)
    xb, yb = b.deserialize(x.serialize()), b.deserialize(y.serialize())
    assert np.array_equal(b.decrypt(xb), a.decrypt(x))
    assert np.array_equal(b.multiply(xb, yb).to_host(), a.multiply(x, y).to_host())
    assert np.array_equal(b.rotate(xb, -2).to_host(), a.rotate(x, -2).to_host())
    sa = a.to_shared(a.encrypt(_z(rng, 4, 64), 2.0 ** 40, 4), 2)
    sb = b.deserialize(sa.serialize())
    assert np.array_equal(b.rotate(sb, 1).to_host(), a.rotate(sa, 1).to_host())
    assert np.array_equal(b.from_shared(sb).to_host(), a.from_shared(sa).to_host())
    assert np.array_equal(b.decrypt(sb), a.decrypt(sa))
    # the stream: secret (1 + 2 auxiliary), relin, 2 Galois, format, 2 backward, 2 Sh-Galois, end
    kinds = [r[0][2] for r in _records(open(path, "rb").read())]
    assert kinds == [3, 4, 5, 5, 7, 8, 8, 6, 6, 9]


def test_keys_without_secrets_and_damaged_streams(tmp_path):
    a, c = _host(seed=11), _host(seed=5)
    a.gen_relin_key()
    a.gen_galois_keys([a.galois_elt(3)])
    path = str(tmp_path / "pub.bin")
    a.save_keys(path, with_secrets=False)
    blob = open(path, "rb").read()
    assert [r[0][2] for r in _records(blob)] == [4, 5, 9]
    c.load_keys(path)
    x = a.encrypt(_z(np.random.default_rng(4), 1, 32), 2.0 ** 40, 4)
    xc = c.deserialize(x.serialize())
    assert np.array_equal(c.rotate(xc, 3).to_host(), a.rotate(x, 3).to_host())
    assert np.abs(c.decrypt(xc) - a.decrypt(x)).max() > 1e-2  # the secret did not move
    cut = str(tmp_path / "cut.bin")
    open(cut, "wb").write(blob[:-HEADER.size - 8])  # no end record
    d = _host(seed=6)
    with pytest.raises(HostError, match="truncated"):
        d.load_keys(cut)
    bad = bytearray(blob)
    bad[HEADER.size + 8 * 5] ^= 0x10
    open(cut, "wb").write(bytes(bad))
    with pytest.raises(HostError, match="digest|prime"):
        d.load_keys(cut)


def test_secret_text_is_the_reference_format(tmp_path):
    """A ternary secret written as the reference's text file from the oracle's NTT (the
    reference's twiddles and bit-reversed order) is the host's secret after import."""
    primes = _primes()
    o = O.Oracle(LOG_N, primes, len(primes) - NP, NP)
    rng = np.random.default_rng(5)
    n = 1 << LOG_N
    s = np.zeros(n, dtype=np.int64)
    pos = rng.choice(n, 64, replace=False)
    s[pos] = rng.choice([-1, 1], 64)
    res = np.stack([np.where(s < 0, q + s, s).astype(np.uint64) % np.uint64(q) for q in primes])
    ntt = o.ntt(res[None])[0]
    text = tmp_path / "sk.txt"
    text.write_text("\n".join(str(int(v)) for v in ntt.ravel()) + "\n")
    a, b = _host(seed=11), _host(seed=12)
    a.import_secret_text(str(text))
    b.import_secret_text(str(text))
    x = a.encrypt(_z(rng, 1, 64), 2.0 ** 40, 4)
    assert np.abs(b.decrypt(b.deserialize(x.serialize())) - a.decrypt(x)).max() == 0
    out = tmp_path / "sk_out.txt"
    a.export_secret_text(str(out))
    assert out.read_text() == text.read_text()
    # damaged text files
    lines = text.read_text().split("\n")
    for i, edit, msg in [(3, "12x", "trailing"), (5, "abc", "not a number"), (0, str(primes[0]), "below its prime"),
                         (n + 1, str((int(lines[n + 1]) + 1) % primes[1]), "small integer")]:
        bad = list(lines)
        bad[i] = edit
        p = tmp_path / "bad.txt"
        p.write_text("\n".join(bad))
        with pytest.raises(HostError, match=msg):
            a.import_secret_text(str(p))
    (tmp_path / "short.txt").write_text("\n".join(lines[:-10]))
    with pytest.raises(HostError, match="expected"):
        a.import_secret_text(str(tmp_path / "short.txt"))


def test_import_key_in_the_reference_layout(tmp_path):
    """A relinearisation key and a Galois key given as raw [dnum][2][QP][N] words (the
    reference's key digits) behave as the generated ones."""
    a, b = _host(seed=11), _host(seed=12)
    a.gen_relin_key()
    e = a.galois_elt(5)
    a.gen_galois_keys([e])
    a.save_keys(str(tmp_path / "k.bin"), with_secrets=False)
    recs = _records(open(tmp_path / "k.bin", "rb").read())
    relin = next(r[1] for r in recs if r[0][2] == 4)
    gal = next(r[1] for r in recs if r[0][2] == 5)
    b.import_key(relin)
    b.import_key(gal, elt=e)
    rng = np.random.default_rng(6)
    x, y = a.encrypt(_z(rng, 1, 32), 2.0 ** 40, 6), a.encrypt(_z(rng, 1, 32), 2.0 ** 40, 6)
    xb, yb = b.deserialize(x.serialize()), b.deserialize(y.serialize())
    assert np.array_equal(b.multiply(xb, yb).to_host(), a.multiply(x, y).to_host())
    assert np.array_equal(b.rotate(xb, 5).to_host(), a.rotate(x, 5).to_host())
    with pytest.raises(HostError, match="expected"):
        b.import_key(relin[:-1])
    bad = relin.copy()
    bad[3] = a.primes[0]
    with pytest.raises(HostError, match="below its prime"):
        b.import_key(bad)
    with pytest.raises(HostError, match="Galois element"):
        b.import_key(gal, elt=4)


@pytest.mark.gpu
def test_records_are_the_same_bytes_in_both_builds(tmp_path):
    """Keys and ciphertexts written by the CUDA build equal the oracle build's byte for byte,
    and a record from either build loads in the other."""
    import shmoai_b200.host as H

    primes = _primes()
    cu, orc = _host(seed=21, lib=H.PRODUCT_LIB, primes=primes), _host(seed=21, primes=primes)
    for h in (cu, orc):
        h.gen_relin_key()
        h.gen_galois_keys([h.galois_elt(1)])
        h.gen_shared_keys(2, [h.galois_elt(1)], hamming_weight=64)
    pc, po = str(tmp_path / "cu.bin"), str(tmp_path / "orc.bin")
    cu.save_keys(pc)
    orc.save_keys(po)
    assert open(pc, "rb").read() == open(po, "rb").read()
    rng = np.random.default_rng(7)
    z = _z(rng, 2, 64)
    x_cu, x_orc = cu.encrypt(z, 2.0 ** 40, 5), orc.encrypt(z, 2.0 ** 40, 5)
    assert x_cu.serialize() == x_orc.serialize()
    other = _host(seed=33, lib=H.PRODUCT_LIB, primes=primes)
    other.load_keys(po)
    xo = other.deserialize(x_orc.serialize())
    assert np.array_equal(other.rotate(xo, 1).to_host(), orc.rotate(x_orc, 1).to_host())
    assert np.array_equal(other.decrypt(xo), orc.decrypt(x_orc))
