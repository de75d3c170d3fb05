"""The reference-side binding shown in INTEGRATION.md compiles against the
upstream headers (Input_Reader.h, Cutoff_Wins.h) and include/cicy_b200.h.

The C++ block that opens with a file comment (the maintainer's Gpu_Path.h) is
cut out of the document and compiled with `g++ -fsyntax-only`, the way the
upstream sources are compiled for the oracle (oracle/Makefile: C++11 with the
forced-include compatibility header).  Needs the upstream tree
(CICY_REF_DIR); skipped without it.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.environ.get("CICY_REF_DIR", "/root/reference")


def _binding_blocks():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, flags=re.S)
    return [b for b in blocks if b.lstrip().startswith("//") and "#include" in b]


def test_binding_block_present():
    blocks = _binding_blocks()
    assert len(blocks) >= 1
    assert "cicy_upload_network" in blocks[0] and "cicy_params" in blocks[0]


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "Input_Reader.h")), reason="upstream tree not present")
@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_binding_compiles_against_upstream_headers(tmp_path):
    for k, block in enumerate(_binding_blocks()):
        src = tmp_path / f"binding_{k}.cpp"
        src.write_text("#include <stdexcept>\n" + block + "\nint main() { return 0; }\n")
        cmd = ["g++", "-std=c++11", "-fsyntax-only", "-w", "-include", os.path.join(ROOT, "oracle", "ref_compat.h"),
               "-I", os.path.join(ROOT, "include"), "-I", REF_DIR, str(src)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]
