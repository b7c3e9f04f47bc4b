"""The INTEGRATION.md section 2 bridge, compiled and checked on the CPU.

The ```cpp block of section 2 is extracted verbatim into b200_bridge.cpp and
compiled by nvcc with tests/bridge/check_bridge.cu against the reference's
own CudaPayload (noor/header/payload.h), CudaHosekSky, CudaCamera and
CudaSpec (noor/cuda/*.cuh, through the oracle's prelude standing in for
path_tracer.cuh).  The check program fills Noor's objects, runs the bridge's
mirrors and compares every field with the library's structs, then resolves
the library's entry points from the built libnoor_b200.so.  No GPU call is
made.  Needs the reference tree (skipped without it).
"""
import os
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from oracle.oracle import reference_tree

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "noor_b200" / "libnoor_b200.so"


def bridge_source() -> str:
    text = (ROOT / "INTEGRATION.md").read_text()
    sec = text[text.index("## 2."):text.index("## 3.")]
    blocks = re.findall(r"```cpp\n(.*?)```", sec, re.S)
    assert len(blocks) == 1
    return blocks[0]


def test_bridge_block_is_complete():
    src = bridge_source()
    # no elided rows or lines
    assert "/* ..." not in src and not re.search(r"^\s*\.\.\.", src, re.M)
    for name in ("load_cuda_data", "update_cuda_camera", "update_cuda_hosek", "update_cuda_spec",
                 "cuda_path_tracer", "debug_skydome", "device_free_memory", "get_lookAt"):
        assert re.search(r"^void %s\(" % name, src, re.M), name


def test_bridge_compiles_against_the_reference_and_mirrors_every_field(tmp_path):
    noor = reference_tree() / "noor"
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not noor.exists():
        pytest.skip("reference tree not present")
    if not Path(nvcc).exists():
        pytest.skip("nvcc not found")
    if not LIB.exists():
        pytest.skip("libnoor_b200.so not built")
    (tmp_path / "b200_bridge.cpp").write_text(bridge_source())
    shutil.copy(ROOT / "tests" / "bridge" / "path_tracer.cuh", tmp_path / "path_tracer.cuh")
    exe = tmp_path / "check_bridge"
    cmd = [nvcc, "-std=c++17", "-w", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", str(tmp_path), "-I", str(ROOT / "oracle" / "refdev" / "shim"), "-I", str(ROOT / "oracle" / "refdev"),
           "-I", str(noor / "cuda"), "-I", str(noor / "header"), "-I", str(ROOT / "oracle" / "ref_shim"),
           "-I", str(ROOT / "include"), str(ROOT / "tests" / "bridge" / "check_bridge.cu"), "-o", str(exe), "-ldl"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-4000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60,
                         env=dict(os.environ, NOOR_B200_LIB=str(LIB)))
    assert run.returncode == 0 and "bridge ok" in run.stdout, run.stdout + run.stderr
