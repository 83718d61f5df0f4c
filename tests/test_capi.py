"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute call: this runs without a GPU)."""
import glob
import os
import re

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(shm_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"shm_context_create", "shm_ntt_forward", "shm_keyswitch", "shm_rotate", "shm_ctpt_matmul"} <= names


def test_library_exports_every_declared_symbol():
    import shmoai_b200

    lib = shmoai_b200.lib()
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_last_error_without_gpu_work():
    import shmoai_b200

    lib = shmoai_b200.lib()
    assert lib.shm_last_error() is not None
