"""The N > 1 path on CPU: two gloo ranks each bootstrap their shard of a batch through
the host library's oracle build (N = 2^12) and gather the results on rank 0, which
must equal the single-process bootstrap of the whole batch bit for bit (ciphertexts
are independent units, so sharding needs no collective on the data path)."""
import os
import socket

import numpy as np
import pytest

from shmoai_b200.shard import gather_to_rank0, max_over_ranks, shard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_HOST = os.path.join(ROOT, "oracle", "_build", "libshmoai_host_oracle.so")
SMALL_BITS = [51] + [46] * 6 + [51] * 13 + [51] * 5


def test_shard_bounds():
    assert [shard(10, r, 3) for r in range(3)] == [(0, 4), (4, 3), (7, 3)]
    assert [shard(16, r, 3, unit=4) for r in range(3)] == [(0, 8), (8, 4), (12, 4)]
    assert sum(shard(768, r, 8, unit=8)[1] for r in range(8)) == 768
    with pytest.raises(ValueError):
        shard(10, 0, 2, unit=4)


def _setup(members):
    from oracle import oracle as O
    from shmoai_b200.host import Bootstrapper, Host

    h = Host(12, O.gen_primes(12, SMALL_BITS), 5, hamming_weight=64, seed=31, lib=ORACLE_HOST)
    h.gen_relin_key()
    bs = Bootstrapper(h, 2.0 ** 46, 4)
    if members:
        h.gen_shared_keys(members, bs.galois_elts(), hamming_weight=64)
    else:
        h.gen_galois_keys(bs.galois_elts())
    rng = np.random.default_rng(8)
    z = rng.uniform(-1, 1, (4, h.n // 2)) + 1j * rng.uniform(-1, 1, (4, h.n // 2))
    return h, bs, z


def _rank(rank, world, port, members, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        h, bs, z = _setup(members)
        start, count = shard(len(z), rank, world, unit=members or 1)
        ct = h.encrypt(z, 2.0 ** 46, 4)  # the same ciphertexts as the single process
        mine = h.ct_from_host(ct.to_host()[start:start + count], ct.scale)
        out = bs.run(mine, members=members)
        t = max_over_ranks(float(rank + 1), dist)
        got = gather_to_rank0(out.to_host(), dist)
        if rank == 0:
            q.put((t, np.concatenate(got)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("members", [0, 2])
def test_two_gloo_ranks_match_one_process(members):
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, members, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, sharded = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert t == 2.0  # max over ranks
    h, bs, z = _setup(members)
    whole = bs.run(h.encrypt(z, 2.0 ** 46, 4), members=members).to_host()
    assert np.array_equal(sharded, whole)
