"""MOAI driver code compiled unchanged against include/moai_shim.hpp (the reference's moai:: and
PhantomFHE names over the C++ host library): the config-2 driver of
src/include/test/matrix_mul/test_ct_pt_matrix_mul.cuh:7-169 restated in tests/shim/ctpt_driver.cpp
(closed form (j + 1) * num_col / 128 per token row j), and evaluator calls in tests/shim/ops_driver.cpp.
CPU: linked against the oracle build of the host library at reduced sizes.  GPU: linked against the
CUDA build at the reference test's own sizes (N = 2^16, 256 inputs x 128 tokens, 768 -> 64)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_BUILD = os.path.join(ROOT, "oracle", "_build")
CUDA_BUILD = os.path.join(ROOT, "shmoai_b200", "_build")


def _build(tmp_path, name, libdir, libs):
    exe = str(tmp_path / name)
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "shim", name + ".cpp"), "-L" + libdir] + ["-l" + x for x in libs] + \
          ["-Wl,-rpath," + libdir, "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def _run(exe, *args):
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_ctpt_driver_on_oracle(tmp_path):
    exe = _build(tmp_path, "ctpt_driver", ORACLE_BUILD, ["shmoai_host_oracle", "shmoai_oracle_capi"])
    out = _run(exe, 12, 16, 128, 96, 8)
    # 16 primes, the product rescaled once: chain index 2, 14 limbs, scale reset to 2^40
    assert "chain_index 2 coeff_modulus_size 14 scale_log2 40.000" in out, out


def test_ops_driver_on_oracle(tmp_path):
    exe = _build(tmp_path, "ops_driver", ORACLE_BUILD, ["shmoai_host_oracle", "shmoai_oracle_capi"])
    assert _run(exe, 12).strip().endswith("ok")


@pytest.mark.gpu
def test_ctpt_driver_reference_sizes_on_b200(tmp_path):
    exe = _build(tmp_path, "ctpt_driver", CUDA_BUILD, ["shmoai_host", "shmoai_b200"])
    out = _run(exe, 16, 256, 128, 768, 64)
    assert "chain_index 2 coeff_modulus_size 14 scale_log2 40.000" in out, out


@pytest.mark.gpu
def test_ops_driver_on_b200(tmp_path):
    exe = _build(tmp_path, "ops_driver", CUDA_BUILD, ["shmoai_host", "shmoai_b200"])
    assert _run(exe, 16).strip().endswith("ok")
