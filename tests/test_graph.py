"""CUDA graphs of whole operation sequences: shm_graph_* (include/shmoai_ckks.h) and
shmoai::Graph / BatchBootstrapper::capture (include/shmoai/host.hpp).

CPU: the oracle's C ABI refuses graphs with a clear error (host arithmetic has nothing to
record).  GPU: a replayed graph gives the eager results bit for bit, also for new inputs
written between launches, and adds its kernels to the launch counter.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_CAPI = os.path.join(ROOT, "oracle", "_build", "libshmoai_oracle_capi.so")
SMALL_BITS = [51] + [46] * 6 + [51] * 13 + [51] * 5  # N = 2^12, nq = 20, np = 5
DELTA = 2.0 ** 46


def test_oracle_abi_refuses_graphs():
    lib = ctypes.CDLL(ORACLE_CAPI)
    lib.shm_last_error.restype = ctypes.c_char_p
    lib.shm_graph_begin.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.shm_graph_end.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    lib.shm_graph_launch.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.shm_graph_kernels.restype = ctypes.c_uint64
    lib.shm_graph_kernels.argtypes = [ctypes.c_void_p]
    token = ctypes.c_char()
    assert lib.shm_graph_begin(None, ctypes.byref(token)) != 0
    assert b"CUDA graphs need the CUDA library" in lib.shm_last_error()
    g = ctypes.c_void_p(1)
    assert lib.shm_graph_end(None, ctypes.byref(token), ctypes.byref(g)) != 0 and not g.value
    assert lib.shm_graph_launch(None, None) != 0
    assert lib.shm_graph_kernels(None) == 0


@pytest.mark.gpu
def test_kernel_graph_replays_a_primitive_chain_bit_exact():
    """NTT inverse + forward, a rotation, multiply, relinearisation and rescale recorded
    once and replayed for two different inputs."""
    import torch

    import shmoai_b200
    from shmoai_b200.ckks import CKKSContext

    bits = [60] + [50] * 7 + [60] * 4  # nq = 8, np = 4, dnum = 2
    ctx = CKKSContext(16, bits=bits, n_special=4)
    n, L, QP, dnum = ctx.n, ctx.nq, ctx.nq + ctx.np, ctx.dnum
    B = 2
    g = torch.Generator(device="cuda").manual_seed(77)
    pt = torch.tensor(ctx.primes.astype(np.int64), device="cuda")

    def residues(shape, primes):
        x = torch.randint(0, 2 ** 62, shape, device="cuda", generator=g, dtype=torch.int64)
        return torch.remainder(x, primes.view(*([1] * (len(shape) - 2)), -1, 1))

    x1, x2 = residues((B, 2, L, n), pt[:L]), residues((B, 2, L, n), pt[:L])
    ct2 = residues((B, 2, L, n), pt[:L])
    gk, rk = residues((dnum, 2, QP, n), pt), residues((dnum, 2, QP, n), pt)
    ws = torch.empty(max(ctx.workspace_bytes("keyswitch", B, L) // 8 + B * 2 * L * n,
                         ctx.workspace_bytes("rescale", 2 * B, L) // 8), dtype=torch.int64, device="cuda")
    src, work, rot = torch.empty_like(x1), torch.empty_like(x1), torch.empty_like(x1)
    m = torch.empty(B, 3, L, n, dtype=torch.int64, device="cuda")
    rel, out = torch.empty_like(x1), torch.empty(B, 2, L - 1, n, dtype=torch.int64, device="cuda")

    def chain():
        work.copy_(src)
        ctx.ntt_inverse_(work)
        ctx.ntt_forward_(work)
        ctx.rotate(work, 1, gk, out=rot, workspace=ws)
        ctx.multiply(rot, ct2, out=m)
        ctx.relinearize(m, rk, out=rel, workspace=ws)
        ctx.rescale(rel, out=out, workspace=ws)

    eager = []
    for x in (x1, x2):
        src.copy_(x)
        chain()
        eager.append(out.clone())
    graph = ctx.capture(chain)
    assert graph.kernels >= 10
    lib = shmoai_b200.lib()
    for x, want in zip((x1, x2), eager):
        src.copy_(x)
        out.zero_()
        l0 = lib.shm_kernel_launches()
        graph.launch()
        torch.cuda.synchronize()
        assert lib.shm_kernel_launches() - l0 == graph.kernels
        assert torch.equal(out, want)
    graph.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("members", [0, 2])
def test_bootstrap_graph_matches_eager_bit_exact(members):
    from shmoai_b200.host import Bootstrapper, Host

    h = Host(12, O.gen_primes(12, SMALL_BITS), 5, hamming_weight=64, seed=31)
    h.gen_relin_key()
    bs = Bootstrapper(h, DELTA, 4)
    if members:
        h.gen_shared_keys(members, bs.galois_elts(), hamming_weight=64)
    else:
        h.gen_galois_keys(bs.galois_elts())
    rng = np.random.default_rng(8)
    zs = [rng.uniform(-1, 1, (4, h.n // 2)) + 1j * rng.uniform(-1, 1, (4, h.n // 2)) for _ in range(2)]
    cts = [h.encrypt(z, DELTA, 4) for z in zs]
    want = [bs.run(c, members=members).to_host() for c in cts]
    inp = h.encrypt(zs[0], DELTA, 4)
    graph, out = bs.capture(inp, members=members)
    assert graph.kernels > 100
    for c, z, w in zip(cts, zs, want):
        data = c.to_host()
        inp.write_from_ptr(data.ctypes.data)
        graph.launch()
        got = out.to_host()
        assert np.array_equal(got, w)
        assert np.abs(h.decrypt(out) - z).mean() < 2e-5
    graph.close()
