"""Turns the output of the reference golden harness into the committed fixtures.

How the fixtures in this folder were made:

1. ``oracle/build_ref.sh`` compiles the reference evaluator (ShMOAI's vendored
   PhantomFHE + the moai:: adapter) for sm_100a together with
   ``oracle/ref_golden.cu`` into ``oracle/_ref/ref_golden``.
2. On a B200: ``oracle/_ref/ref_golden <tiny|prim|boot> > raw_<set>.json``.
   The reference prints one debug line of its own into stdout during key
   generation (thirdparty/phantom-fhe/src/secretkey.cu:461).
3. ``python tests/golden/make_golden.py raw_tiny.json raw_prim.json raw_boot.json``
   drops every line that is not part of the JSON document, validates it and
   writes ``golden_<set>.json`` here.

Inputs and key material of every record are rebuilt by the tests with
``oracle.oracle.fill`` (the same counter generator the harness used), so the
fixtures only carry checksums and the first coefficients of each limb.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def clean(path):
    lines = open(path).read().splitlines()
    keep = [ln for ln in lines if ln[:1] in ("{", "}", " ") or ln == ""]
    doc = json.loads("\n".join(keep))
    name = doc["params"]["name"]
    out = os.path.join(HERE, f"golden_{name}.json")
    with open(out, "w") as f:
        json.dump(doc, f, separators=(",", ":"))
    return out


if __name__ == "__main__":
    for p in sys.argv[1:]:
        print(clean(p))
