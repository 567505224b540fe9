"""The Sirius adapter (adapter/sirius_hash_join_sj.cpp), compiled and RUN: it is linked with the
stand-in cuDF / RMM classes (adapter/standin + tests/adapter_host/standin_runtime.cpp), libsj.so
and the CUDA runtime under AddressSanitizer, and driven over the reference's NULL-join fixture
(test/cpp/integration/test_gpu_execution_join_nulls.cpp:37-104) and the operator-level MARK cases
(test/cpp/operator/test_physical_mark_join.cpp:245-530), restated in tests/golden/.

Every table is built, probed and destroyed through sj_hash_table, so each destructor frees through
the allocator context the table was built with (a context that must outlive the table; ASan's
stack-use-after-return detection reports it otherwise). The RIGHT family runs with the sides
swapped, as the reference's STANDARD mode does (src/op/sirius_physical_hash_join.cpp:1879-1895).
An allocation-refusal sweep refuses the Nth device allocation of a build + probe for every N: each
refusal must come out as rmm::out_of_memory (the operator's OOM-reschedule path,
src/pipeline/gpu_pipeline_task.cpp:386-437) with nothing left allocated."""
import json
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HOST = ROOT / "tests" / "adapter_host"
EXE = HOST / "_build" / "run_fixture"
CUDA_LIB = Path("/usr/local/cuda/lib64")

GOLD = json.loads((ROOT / "tests" / "golden" / "join_known_answers.json").read_text())


def _compile(built):
    EXE.parent.mkdir(exist_ok=True)
    cmd = ["g++", "-std=c++20", "-g", "-O1", "-fsanitize=address", "-fno-omit-frame-pointer",
           "-Wall", "-Wextra", "-Werror",
           f"-I{ROOT / 'adapter' / 'standin'}", f"-I{ROOT / 'adapter'}", f"-I{ROOT / 'include'}", f"-I{HOST}",
           str(ROOT / "adapter" / "sirius_hash_join_sj.cpp"), str(HOST / "standin_runtime.cpp"),
           str(HOST / "run_fixture.cpp"),
           f"-L{ROOT / 'sirius_b200'}", "-lsj", f"-L{CUDA_LIB}", "-lcudart",
           f"-Wl,-rpath,{ROOT / 'sirius_b200'}", f"-Wl,-rpath,{CUDA_LIB}", "-o", str(EXE)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return EXE


def _fixture_input() -> str:
    f = GOLD["nulls_fixture"]
    side = lambda s: " ".join(f"{i}:{'N' if k is None else k}" for i, k in zip(f[s]["id"], f[s]["k"]))
    keys = lambda v: ",".join("N" if k is None else str(k) for k in v) if v else "-"
    lines = [f"L {side('l')}", f"R {side('r')}"]
    for c in GOLD["mark_cases"]:
        lines.append(f"M {c['name'].replace(' ', '_')} {keys(c['left'])} {keys(c['right'])}")
    return "\n".join(lines) + "\n"


def _rows(v):
    """Canonical order of result rows (NULL sorts first)."""
    key = lambda r: tuple((0, 0) if x is None else (1, x) for x in (r if isinstance(r, list) else [r]))
    return sorted([r if isinstance(r, list) else [r] for r in v], key=key)


needs_gxx = pytest.mark.skipif(shutil.which("g++") is None or not (CUDA_LIB / "libcudart.so").exists(),
                               reason="needs g++ and the CUDA runtime library")


@needs_gxx
def test_adapter_links_with_libsj(built):
    """The adapter, the stand-in runtime and the fixture driver compile and link (no GPU)."""
    assert _compile(built).exists()


@pytest.mark.gpu
@needs_gxx
def test_adapter_runs_known_answers_under_asan(cuda):
    exe = _compile(True)
    env = dict(os.environ)
    # protect_shadow_gap=0: the CUDA driver maps memory where ASan would otherwise reserve its shadow
    # gap; detect_stack_use_after_return: a dangling allocator context on a returned frame is reported
    env["ASAN_OPTIONS"] = "protect_shadow_gap=0:detect_stack_use_after_return=1:detect_leaks=0:abort_on_error=0"
    r = subprocess.run([str(exe)], input=_fixture_input(), capture_output=True, text=True, env=env, timeout=300)
    assert "AddressSanitizer" not in r.stderr, r.stderr[-4000:]
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-4000:])
    out = {d["case"]: d for d in map(json.loads, r.stdout.strip().splitlines())}
    f = GOLD["nulls_fixture"]
    for case in ("inner", "left", "full", "right", "inner_null_safe"):
        assert _rows(out[case]["rows"]) == _rows(f[case]), case
    assert _rows(out["semi"]["rows"]) == _rows(f["semi"])
    assert _rows(out["anti"]["rows"]) == _rows(f["anti"])
    assert _rows(out["mark_with_null_build"]["rows"]) == _rows(f["mark_with_null_build"])
    # RIGHT_SEMI / RIGHT_ANTI: right rows with / without a left match (r.k 10, 20, 20 match l.k)
    assert _rows(out["right_semi"]["rows"]) == _rows([1, 2, 3])
    assert _rows(out["right_anti"]["rows"]) == _rows([4, 5])
    for c in GOLD["mark_cases"]:
        got = out["mark:" + c["name"].replace(" ", "_")]["rows"]
        assert _rows(got) == _rows([[i, m] for i, m in enumerate(c["mark"])]), c["name"]
    sweep = out["oom_sweep"]
    attempts = sweep["attempts"]
    assert attempts[-1]["outcome"] == "ok:4", attempts[-1]
    assert len(attempts) > 8  # refusals reached the build and the probe, past the input uploads
    for a in attempts[:-1]:
        assert a["outcome"] == "oom", a
    assert all(a["leaked"] == 0 for a in attempts), attempts
    assert sweep["live_allocations"] == 0
