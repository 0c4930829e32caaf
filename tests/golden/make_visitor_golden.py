"""Writes tests/golden/visitor/<query>.sycl: the programs the reference's own code
generator (JITOperatorVisitor::generateCode, src/core/visitor.cpp, after the
Optimizer of src/core/optimizer_rules.cpp) emits for the measured query shapes.

The generator is compiled from the reference sources where they lie by
`make -C oracle visitor` (oracle/visitor/emit_visitor.cpp builds the operator
trees and the catalog of the synthetic schema).  The fixtures let the GPU tests,
which run where the reference is not mounted, feed the reference's codegen
output to cx_compile / cx_execute.  Test infrastructure only.

Usage: python tests/golden/make_visitor_golden.py [reference root]
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent / "visitor"
QUERIES = ["q11", "q31", "q31_nullable", "t0", "t1", "t2", "t3"]


def emitter(ref: Path) -> Path:
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "visitor", f"REF={ref}"], check=True, capture_output=True)
    return ROOT / "oracle" / "_ref" / "emit_visitor"


def emit(binary: Path, query: str) -> str:
    return subprocess.run([str(binary), query], check=True, capture_output=True, text=True).stdout


def main() -> None:
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CRYSTAL_REFERENCE", "/root/reference"))
    binary = emitter(ref)
    OUT.mkdir(exist_ok=True)
    for q in QUERIES:
        (OUT / f"{q}.sycl").write_text(emit(binary, q))
        print(f"wrote {OUT / (q + '.sycl')}")


if __name__ == "__main__":
    main()
