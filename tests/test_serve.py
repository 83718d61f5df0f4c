"""The serving loop (shm_server_*): a mix of rotation batches, a ct-pt matmul and
ordinary and shared-a bootstraps submitted at once onto several slots.  Every result
must equal the same job run alone (bit for bit), queued jobs of the same kind and shape
must be merged into one launch (continuous batching), more than one batch must be in
flight at a time, and a job above the HBM budget is refused at submission.
CPU: the host library's oracle build at N = 2^12; GPU: the CUDA build, additionally
equal to the oracle build bit for bit."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from shmoai_b200.host import Bootstrapper, Host, HostError, Server

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_HOST = os.path.join(ROOT, "oracle", "_build", "libshmoai_host_oracle.so")
SMALL_BITS = [51] + [46] * 6 + [51] * 13 + [51] * 5
DELTA = 2.0 ** 46

# (kind, count, level, step or members); rotations of the same (level, step) can merge
JOBS = [("boot", 2, 4, 0), ("boot", 4, 4, 2), ("mm", 4, 3, 0), ("rot", 3, 5, 1), ("rot", 2, 5, 1),
        ("rot", 1, 4, 3), ("rot", 2, 5, 1)]


def _host(lib):
    h = Host(12, O.gen_primes(12, SMALL_BITS), 5, hamming_weight=64, seed=41, lib=lib)
    h.gen_relin_key()
    bs = Bootstrapper(h, DELTA, 4)
    elts = sorted(set(bs.galois_elts()) | {h.galois_elt(1), h.galois_elt(3)})
    h.gen_galois_keys(elts)
    h.gen_shared_keys(2, bs.galois_elts(), hamming_weight=64)
    return h, bs


def _inputs(h):
    rng = np.random.default_rng(17)
    out = []
    for kind, count, L, _ in JOBS:
        z = rng.uniform(-1, 1, (count, h.n // 2)) + 1j * rng.uniform(-1, 1, (count, h.n // 2))
        scale = DELTA if kind in ("boot", "mm") else 2.0 ** 40
        ct = h.encrypt(z, scale, L)
        out.append((z, ct.to_host(), ct.scale))
    W = np.random.default_rng(3).integers(-(1 << 20), 1 << 20, size=(4, 3), dtype=np.int64)
    return out, W


def _submit(srv, h, inputs, W, i):
    kind, count, L, arg = JOBS[i]
    z, data, scale = inputs[i]
    ct = h.ct_from_host(data, scale)
    if kind == "rot":
        return srv.submit_rotate(ct, arg)
    if kind == "mm":
        return srv.submit_matmul(ct, W, 2.0 ** 20)
    return srv.submit_bootstrap(ct, arg)


def _scenario(lib):
    h, bs = _host(lib)
    inputs, W = _inputs(h)
    alone = []
    srv = Server(h, bs, hbm_budget=64 << 30, slots=1)
    for i in range(len(JOBS)):
        out, _, merged = srv.wait(_submit(srv, h, inputs, W, i))
        assert merged == 1
        alone.append(out.to_host())
    srv.close()
    srv = Server(h, bs, hbm_budget=64 << 30, slots=3)
    srv.pause()  # everything arrives while the slots are busy: the rotations must be merged
    ids = [_submit(srv, h, inputs, W, i) for i in range(len(JOBS))]
    srv.resume()
    mixed, merged, times = [], [], []
    for j in ids:
        out, t, m = srv.wait(j)
        mixed.append(out)
        merged.append(m)
        times.append(t)
    stats = srv.stats()
    srv.close()
    return h, inputs, W, alone, mixed, merged, times, stats


def _check(h, inputs, W, alone, mixed, merged, times, stats):
    for i, (a, m) in enumerate(zip(alone, mixed)):
        assert np.array_equal(a, m.to_host()), f"job {i} {JOBS[i]} differs alone vs in the mix"
    assert stats["jobs"] == len(JOBS) and stats["batches"] < len(JOBS)  # some jobs were merged
    assert max(merged) >= 2
    assert stats["peak_admitted"] <= stats["budget"]
    assert all(s <= b <= e for s, b, e in times)
    # results decrypt to the right values
    for i, (kind, count, L, arg) in enumerate(JOBS):
        z = inputs[i][0]
        got = h.decrypt(mixed[i])
        if kind == "rot":
            assert np.abs(got - np.roll(z, -arg, axis=1)).max() < 1e-5
        elif kind == "boot":
            assert np.abs(got - z).mean() < 2e-5
        else:  # output scale 2^46 * 2^20 / q_2 ~ 2^20 after the (floor) rescale
            want = (W.T.astype(np.float64) / 2.0 ** 20) @ z
            assert np.abs(got - want).max() < 1e-2


def test_serving_mix_equals_jobs_alone_on_oracle():
    res = _scenario(ORACLE_HOST)
    _check(*res)
    assert res[-1]["max_inflight"] >= 2  # batches overlapped


def test_job_above_budget_is_refused():
    h = Host(12, O.gen_primes(12, SMALL_BITS), 5, hamming_weight=64, seed=41, lib=ORACLE_HOST)
    h.gen_galois_keys([h.galois_elt(1)])
    srv = Server(h, None, hbm_budget=1 << 20, slots=1)
    ct = h.encrypt(np.ones((2, 8)), 2.0 ** 40, 5)
    with pytest.raises(HostError, match="above the HBM budget"):
        srv.submit_rotate(ct, 1)
    ct = h.encrypt(np.ones((2, 8)), 2.0 ** 40, 5)
    with pytest.raises(HostError, match="no bootstrapper"):
        srv.submit_bootstrap(ct, 0)
    srv.close()


@pytest.mark.gpu
def test_serving_mix_on_b200_matches_oracle_build():
    g = _scenario(None)
    _check(*g)
    c = _scenario(ORACLE_HOST)
    for i, (a, b) in enumerate(zip(g[4], c[4])):
        assert np.array_equal(a.to_host(), b.to_host()), f"job {i} differs between the CUDA and oracle builds"
