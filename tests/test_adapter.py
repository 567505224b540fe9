"""The Sirius-side adapter (adapter/sirius_hash_join_sj.cpp) compiles against the stand-in
cuDF / RMM declarations of the names it uses (cuDF and RMM are not installed here). No GPU."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_adapter_compiles_against_standin_headers():
    r = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-Wall", "-Wextra", "-Werror",
                        f"-I{ROOT / 'adapter' / 'standin'}", f"-I{ROOT / 'include'}",
                        str(ROOT / "adapter" / "sirius_hash_join_sj.cpp")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_header_is_plain_c():
    """include/sj/sj_join.h is a C header (no C++ or CUDA types in the ABI)."""
    src = ROOT / "include" / "sj" / "sj_join.h"
    r = subprocess.run(["gcc", "-std=c99", "-fsyntax-only", "-Wall", "-Werror", "-x", "c", str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
