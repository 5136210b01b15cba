"""Regenerate tests/golden/primitives.json from make_golden.cpp.

Usage: python tests/golden/make_golden.py
Needs g++ (C++17).  The fixture is committed; this script is how it was made.
"""
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main() -> int:
    with tempfile.TemporaryDirectory() as tmp:
        exe = Path(tmp) / "make_golden"
        subprocess.run(["g++", "-O2", "-std=c++17", str(HERE / "make_golden.cpp"),
                        "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True,
                             text=True).stdout
    (HERE / "primitives.json").write_text(out)
    print(f"wrote {HERE / 'primitives.json'} ({len(out)} bytes)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
