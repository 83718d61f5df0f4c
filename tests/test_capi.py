"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute call: this runs without a GPU)."""
import glob
import os
import re

from conftest import ROOT


def declared_symbols(header=None):
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", header or "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(shm_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"shm_context_create", "shm_ntt_forward", "shm_keyswitch", "shm_rotate", "shm_ctpt_matmul",
            "shm_host_create", "shm_boot_run"} <= names


def test_library_exports_every_declared_symbol():
    import shmoai_b200

    lib = shmoai_b200.lib()
    missing = [n for n in sorted(declared_symbols("shmoai_ckks.h")) if not hasattr(lib, n)]
    assert not missing, missing


def test_host_library_exports_every_declared_symbol():
    from shmoai_b200 import host

    lib = host.load()
    missing = [n for n in sorted(declared_symbols("shmoai_host.h")) if not hasattr(lib, n)]
    assert not missing, missing


def test_oracle_c_abi_covers_what_the_host_library_calls():
    """Every C-ABI function the host library imports exists in the oracle's C ABI, so the
    CPU build of the host pipeline is complete."""
    import subprocess

    host = os.path.join(ROOT, "shmoai_b200", "_build", "libshmoai_host.so")
    capi = os.path.join(ROOT, "oracle", "_build", "libshmoai_oracle_capi.so")
    und = subprocess.run(["nm", "-D", "--undefined-only", host], capture_output=True, text=True).stdout
    need = {ln.split()[-1] for ln in und.splitlines() if ln.split() and ln.split()[-1].startswith("shm_")}
    have = subprocess.run(["nm", "-D", "--defined-only", capi], capture_output=True, text=True).stdout
    have = {ln.split()[-1] for ln in have.splitlines() if ln.split()}
    assert need and not (need - have), sorted(need - have)


def test_last_error_without_gpu_work():
    import shmoai_b200

    lib = shmoai_b200.lib()
    assert lib.shm_last_error() is not None
