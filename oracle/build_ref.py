#!/usr/bin/env python3
"""Build the reference's CUDA sieve program, unmodified except for its run constants.

TEST INFRASTRUCTURE ONLY: the binaries land in oracle/_ref/ (git-ignored) and are run by the
GPU parity tests and bench.py as the reference CUDA baseline; nothing in the product links them.

The reference configures src/voss_v7_live.cu by rewriting three integer constants in its
source before each nvcc build (src/voss_master.py:64-85, values from :114-123).  This script
does the same substitution in memory, writes the patched text to a temporary directory outside
the repository, and compiles it for sm_100a with the reference's own flags (-O3,
src/voss_master.py:138-140).  The reference source is read from its tree and never copied here.

usage: python oracle/build_ref.py [--ref REFERENCE_CHECKOUT] [--n 1000000000 ...]   (--ref defaults to $VOSS_REF)
"""
import argparse
import math
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SEG_NUM = 30_000_000_000  # src/voss_master.py:28 / run_voss.py:25
DEFAULT_NS = [10**9, 10**10, 10**11, 10**12]


def max_pos_for(mem_gb: float, seg_num: int) -> int:
    """MAX_POS sizing of src/voss_master.py:117-123 for a device with mem_gb of memory."""
    needed = max(int(1.5 * seg_num / math.log(seg_num)), 100_000_000)
    budget = 50.0 if mem_gb >= 70 else (20.0 if mem_gb >= 35 else 8.0)
    return min(needed, int(budget * 1e9 / 8))


def patched_source(src: str, n: int, seg: int, max_pos: int) -> str:
    """Replace N, SEG_NUM and MAX_POS integer literals (same targets as voss_master.patch_cuda)."""
    out = re.sub(r"(static\s+const\s+int64_t\s+N\s*=\s*)\d+(;)", rf"\g<1>{n}\g<2>", src)
    out = re.sub(r"(const\s+int64_t\s+SEG_NUM\s*=\s*)\d+(LL)", rf"\g<1>{seg}\g<2>", out)
    out = re.sub(r"(static\s+const\s+int64_t\s+MAX_POS\s*=\s*)\d+(;)", rf"\g<1>{max_pos}\g<2>", out)
    for name, val in (("N", n), ("SEG_NUM", seg), ("MAX_POS", max_pos)):
        if not re.search(rf"int64_t\s+{name}\s*=\s*{val}", out):
            raise RuntimeError(f"could not set {name} in the reference source")
    return out


def binary_name(n: int) -> str:
    return os.path.join(OUT, f"voss_v7_live_{n}")


def build(ref: str, ns, mem_gb: float = 180.0, force: bool = False) -> list:
    src_path = os.path.join(ref, "src", "voss_v7_live.cu")
    if not os.path.exists(src_path):
        raise FileNotFoundError(src_path)
    src = open(src_path, encoding="utf-8").read()
    os.makedirs(OUT, exist_ok=True)
    built = []
    max_pos = max_pos_for(mem_gb, SEG_NUM)
    with tempfile.TemporaryDirectory(prefix="voss_ref_") as tmp:
        for n in ns:
            dst = binary_name(n)
            if os.path.exists(dst) and not force:
                built.append(dst)
                continue
            cu = os.path.join(tmp, f"voss_v7_live_{n}.cu")
            with open(cu, "w", encoding="utf-8") as f:
                f.write(patched_source(src, n, SEG_NUM, max_pos))
            cmd = ["nvcc", "-O3", "-arch=sm_100a", cu, "-o", dst]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("reference build failed:\n" + r.stderr)
            built.append(dst)
    return built


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("VOSS_REF"), required=not os.environ.get("VOSS_REF"))
    ap.add_argument("--n", type=int, nargs="*", default=DEFAULT_NS)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    for b in build(a.ref, a.n, force=a.force):
        print(b)


if __name__ == "__main__":
    sys.exit(main())
