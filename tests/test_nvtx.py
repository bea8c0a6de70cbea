"""NVTX ranges of libvoss.so, on the CPU: a checkpointed run (segments from the oracle) under an
injection library that records the "voss" domain's pushes and pops.  The API call and each
checkpoint write must show as balanced, named ranges, as Nsight Systems would display them."""
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")

CHILD = r"""
import oracle_lib as O
import voss
N, SEG = 600_000, 60_000
voss.run_checkpointed_fn(lambda lo, hi: O.sieve_range(lo, hi, compat=True, seg_num=SEG), N, SEG, True, 2, {d!r})
"""


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    if not os.path.exists(os.path.join(CUDA_INC, "nvtx3", "nvToolsExt.h")):
        pytest.skip("NVTX 3 headers not found")
    so = str(tmp_path_factory.mktemp("nvtx") / "libnvtx_probe.so")
    subprocess.run(["gcc", "-O1", "-shared", "-fPIC", "-I", CUDA_INC, "-o", so, os.path.join(HERE, "nvtx_probe.c")],
                   check=True)
    return so


def test_checkpointed_run_emits_balanced_named_ranges(probe, tmp_path):
    log = tmp_path / "nvtx.log"
    env = dict(os.environ, NVTX_INJECTION64_PATH=probe, VOSS_NVTX_LOG=str(log),
               PYTHONPATH=os.pathsep.join([os.path.join(ROOT, "voss-prime-gaps_v1_b200"), HERE]))
    subprocess.run([sys.executable, "-c", CHILD.format(d=str(tmp_path))], env=env, check=True, timeout=300)
    lines = log.read_text().splitlines()
    assert lines[0] == "domain voss"
    depth, names = 0, []
    for ln in lines[1:]:
        if ln.startswith("push "):
            depth += 1
            names.append((depth, ln[5:]))
        else:
            assert ln == "pop"
            depth -= 1
            assert depth >= 0
    assert depth == 0
    assert names[0] == (1, "voss_run_checkpointed_fn")
    writes = [n for n in names if n[1] == "checkpoint write"]
    assert len(writes) >= 4 and all(dep == 2 for dep, _ in writes)  # 10 segments, one write every 2
