"""Build recipe for the oracle (test infrastructure, never product code).

  oracle/_build/liboracle.so  <- oracle/oracle_*.cpp (this project's CPU
                                 restatement of the reference algorithms)
  oracle/_ref/libvxref.so     <- oracle/ref_shim.cpp compiled against the
                                 reference's own headers, read in place from
                                 <reference>/algorithm/lib/include (only when
                                 that tree is present; nothing is copied);
                                 <reference> is $VX_REFERENCE or ../reference

Usage: python -m oracle.build [--reference PATH]
"""
from __future__ import annotations

import argparse
import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
BUILD = HERE / "_build"
REF_OUT = HERE / "_ref"
LIB = BUILD / "liboracle.so"
REF_LIB = REF_OUT / "libvxref.so"
# The reference checkout: $VX_REFERENCE, else a "reference" directory beside
# this repository.
DEFAULT_REFERENCE = Path(os.environ.get("VX_REFERENCE", str(ROOT.parent / "reference")))
# -O3 without -march=native: the library may run on a different host CPU.
# -ffp-contract=off: every float operation rounds once, as the GPU code's
# explicitly rounded intrinsics do (the ray casts are compared bit for bit).
CXXFLAGS = ["-O3", "-std=c++20", "-ffp-contract=off", "-fPIC", "-shared", "-pthread",
            f"-I{ROOT / 'include'}"]


def _stale(out: Path, srcs: list[Path]) -> bool:
    if not out.exists():
        return True
    deps = srcs + list((ROOT / "include").glob("*.h")) + list(HERE.glob("*.h"))
    return out.stat().st_mtime < max(p.stat().st_mtime for p in deps)


def build_oracle(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(HERE.glob("oracle_*.cpp"))
    if force or _stale(LIB, srcs):
        subprocess.run(["g++", *CXXFLAGS, *map(str, srcs), "-o", str(LIB)],
                       check=True)
    return LIB


def build_reference(reference: Path = DEFAULT_REFERENCE,
                    force: bool = False) -> Path | None:
    inc = reference / "algorithm" / "lib" / "include"
    if not inc.is_dir():
        return None
    REF_OUT.mkdir(exist_ok=True)
    shim = HERE / "ref_shim.cpp"
    if force or _stale(REF_LIB, [shim]):
        subprocess.run(["g++", *CXXFLAGS, f"-I{inc}", str(shim), "-o",
                        str(REF_LIB)], check=True)
    return REF_LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=str(DEFAULT_REFERENCE))
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build_oracle(a.force))
    print(build_reference(Path(a.reference), a.force))
