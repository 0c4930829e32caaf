"""Three-valued filter conditions as the code generator emits them, checked on
the CPU.

The scan kernel evaluates every non-trivial filter leaf as one expression per
row, with `&` / `|` over operands converted to bool (no short-circuit branch).
These tests take the emitted conditions of seeded random predicates over three
nullable int columns, compile them for the host with g++ (with the header's own `db::safe_*`
helpers), and compare the rows they keep,
over every combination of a few values and NULL, with an independent Python
evaluation of SQL's three-valued logic: WHERE keeps a row only when the
predicate is TRUE (AND is FALSE if either side is, OR is TRUE if either side
is, NOT and comparisons of NULL are NULL, IS [NOT] NULL is never NULL).
Reference rules: the emitted 3VL code of `src/core/visitor.cpp` and the truth
table of `test/test_sql_3vl.cpp`.
"""
from __future__ import annotations

import ctypes
import itertools
import os
import random
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from practice_b200 import _lib
from practice_b200.plan import PlanBuilder, Table, and_, case, col, lit, not_, or_, star

COLS = ("qty", "price", "disc")
VALUES = (-2, 0, 1, 3, 5)
PREFIX = "flags[i] = (tid + BLOCK_THREADS * i < num_tile_items) ? ((int)(flags[i] != 0) & (int)(bool)("
SUFFIX = ")) : flags[i];"

HEADER = Path(__file__).resolve().parent.parent / "practice_b200" / "csrc" / "crystal_sm100.cuh"


def _host_safe_helpers() -> str:
    """The `db::safe_*` helpers of the shipped header (its integer part, up to
    the atomics), compiled for the host."""
    src = HEADER.read_text()
    i = src.index("namespace db {")
    j = src.index("CX_DEVICE unsigned long long bit_cast_double_to_ull", i)
    return "#include <cstdint>\n#define CX_DEVICE static inline\n" + src[i:j] + "}  // namespace db\n"


# ------------------------------------------------------------ random predicates

def _value(rng: random.Random, depth: int):
    r = rng.random()
    if depth <= 0 or r < 0.45:
        return col(rng.choice(COLS))
    if r < 0.65:
        return lit(rng.choice(VALUES))
    if r < 0.85:
        return getattr(_value(rng, depth - 1), rng.choice(("__add__", "__sub__", "__mul__")))(_value(rng, depth - 1))
    return case(_pred(rng, depth - 1), _value(rng, depth - 1), _value(rng, depth - 1))


def _pred(rng: random.Random, depth: int):
    r = rng.random()
    if depth <= 0 or r < 0.35:
        if rng.random() < 0.25:
            v = _value(rng, 1)
            return v.is_null() if rng.random() < 0.5 else v.not_null()
        return getattr(col(rng.choice(COLS)), rng.choice(("eq", "ne", "lt", "le", "gt", "ge")))(_value(rng, 1))
    if r < 0.6:
        return and_(_pred(rng, depth - 1), _pred(rng, depth - 1))
    if r < 0.85:
        return or_(_pred(rng, depth - 1), _pred(rng, depth - 1))
    return not_(_pred(rng, depth - 1))


# ------------------------------------------------------ three-valued evaluation

def _eval(e, row):
    """Value of expression `e` on `row` ({col: int or None}); None is NULL."""
    op = e.op
    if op == "col":
        return row[e.name]
    if op == "int":
        return e.val
    if op in ("add", "sub", "mul"):
        x, y = _eval(e.kids[0], row), _eval(e.kids[1], row)
        if x is None or y is None:
            return None
        return x + y if op == "add" else x - y if op == "sub" else x * y
    if op in ("eq", "ne", "lt", "le", "gt", "ge"):
        x, y = _eval(e.kids[0], row), _eval(e.kids[1], row)
        if x is None or y is None:
            return None
        return {"eq": x == y, "ne": x != y, "lt": x < y, "le": x <= y, "gt": x > y, "ge": x >= y}[op]
    if op == "and":
        x, y = _eval(e.kids[0], row), _eval(e.kids[1], row)
        if x is False or y is False:
            return False
        return None if x is None or y is None else True
    if op == "or":
        x, y = _eval(e.kids[0], row), _eval(e.kids[1], row)
        if x is True or y is True:
            return True
        return None if x is None or y is None else False
    if op == "not":
        x = _eval(e.kids[0], row)
        return None if x is None else not x
    if op in ("isnull", "notnull"):
        x = _eval(e.kids[0], row)
        return (x is None) if op == "isnull" else (x is not None)
    if op == "case":
        c = _eval(e.kids[0], row)
        return _eval(e.kids[1], row) if c is True else _eval(e.kids[2], row)
    raise AssertionError(f"unexpected op {op}")


# ------------------------------------------------------------------- harness

def _conditions(pred) -> list[str]:
    """The emitted filter conditions of a plan filtering on `pred` (one per
    conjunct the generator splits off; the scan keeps a row when all hold)."""
    t = {"T": Table("T", list(COLS), 1000, fact=True)}
    b = PlanBuilder(t, "T", nullable=set(COLS), name="filter3vl")
    b.filter(pred)
    plan = b.aggregate([], [("count", star())])
    src = _lib.codegen(plan.text())
    conds = []
    for line in src.splitlines():
        s = line.strip()
        if s.startswith(PREFIX):
            assert s.endswith(SUFFIX), s
            conds.append(s[len(PREFIX):-len(SUFFIX)])
    assert "BlockPredA" not in src  # every column is nullable: no two-valued fast path
    return conds


def _compile(funcs: list[list[str]], tmp_path) -> ctypes.CDLL:
    body = [_host_safe_helpers()]
    for k, conds in enumerate(funcs):
        body.append(f'extern "C" void eval_{k}(int n, const int* A, const int* AV, const int* B, const int* BV, '
                    "const int* C, const int* CV, int* out) {")
        body.append("  for (int r = 0; r < n; ++r) {")
        body.append("    const int i = 0;")
        body.append("    int qty[1] = {A[r]}, qty_valid[1] = {AV[r]}, price[1] = {B[r]}, price_valid[1] = {BV[r]};")
        body.append("    int disc[1] = {C[r]}, disc_valid[1] = {CV[r]};")
        body.append("    (void)qty; (void)qty_valid; (void)price; (void)price_valid; (void)disc; (void)disc_valid; (void)i;")
        body.append("    int keep = 1;")
        for cond in conds:
            body.append(f"    keep &= (int)(bool)({cond});")
        body.append("    out[r] = keep;")
        body.append("  }")
        body.append("}")
    cpp = tmp_path / "filters.cpp"
    so = tmp_path / "libfilters.so"
    cpp.write_text("\n".join(body) + "\n")
    gxx = shutil.which("g++") or "/usr/bin/g++"
    subprocess.run([gxx, "-O1", "-std=c++17", "-shared", "-fPIC", "-o", str(so), str(cpp)], check=True)
    return ctypes.CDLL(str(so))


def _grid():
    """Every combination of VALUES or NULL for the three columns (a NULL's
    value word holds garbage, as in a real column: two different ones)."""
    per_col = [(v, 1) for v in VALUES] + [(3, 0), (-2, 0)]
    rows = list(itertools.product(per_col, repeat=len(COLS)))
    arrs = []
    for j in range(len(COLS)):
        arrs.append(np.array([r[j][0] for r in rows], dtype=np.int32))
        arrs.append(np.array([r[j][1] for r in rows], dtype=np.int32))
    py_rows = [{c: (r[j][0] if r[j][1] else None) for j, c in enumerate(COLS)} for r in rows]
    return arrs, py_rows


@pytest.mark.skipif(shutil.which("g++") is None and not os.path.exists("/usr/bin/g++"),
                    reason="needs a host C++ compiler")
def test_emitted_filters_follow_three_valued_logic(tmp_path):
    rng = random.Random(20241204)
    preds = [_pred(rng, 3) for _ in range(80)]
    funcs = [_conditions(p) for p in preds]
    for conds in funcs:
        for cond in conds:
            assert "&&" not in cond and "||" not in cond, cond  # evaluated without short-circuit branches
    lib = _compile(funcs, tmp_path)
    arrs, py_rows = _grid()
    n = len(py_rows)
    ptr = ctypes.POINTER(ctypes.c_int)
    out = np.zeros(n, dtype=np.int32)
    kept_any = dropped_any = 0
    for k, p in enumerate(preds):
        fn = getattr(lib, f"eval_{k}")
        fn.argtypes = [ctypes.c_int] + [ptr] * 7
        fn(n, *[x.ctypes.data_as(ptr) for x in arrs], out.ctypes.data_as(ptr))
        want = np.array([_eval(p, r) is True for r in py_rows], dtype=np.int32)
        bad = np.nonzero(out != want)[0]
        assert bad.size == 0, f"{p.sexpr()}: row {py_rows[bad[0]]} kept={out[bad[0]]} want={want[bad[0]]}"
        kept_any += int(want.any())
        dropped_any += int((want == 0).any())
    assert kept_any > 20 and dropped_any > 20  # the predicates are not trivially constant


@pytest.mark.parametrize("name", ["a", "flags", "tid", "hash", "int", "threadIdx", "BlockLoad", "gt3", "x5_", "h0_1",
                                  "acc_2", "__x", "atomicAdd", "2col", "lo-rev"])
def test_column_names_that_collide_with_generated_identifiers_are_rejected(name):
    """A column name that the generated kernels already use (or that is not a
    C identifier) would make NVRTC fail with an unrelated message; the plan
    reader rejects it and names the column."""
    t = {"T": Table("T", ["lo_quantity", name], 1000, fact=True)}
    plan = PlanBuilder(t, "T", name="reserved").aggregate([], [("count", star())])
    with pytest.raises(_lib.CxError) as e:
        _lib.codegen(plan.text())
    assert e.value.code == -1 and name in str(e.value)  # CX_E_INVALID


def test_validity_register_collision_is_rejected_and_plain_names_compile():
    t = {"T": Table("T", ["qty", "qty_valid"], 1000, fact=True)}
    plan = PlanBuilder(t, "T", nullable={"qty"}, name="v").filter(col("qty").gt(lit(1))).aggregate(
        [], [("count", star())])
    with pytest.raises(_lib.CxError, match="qty_valid"):
        _lib.codegen(plan.text())
    t = {"T": Table("T", list(COLS), 1000, fact=True)}
    plan = PlanBuilder(t, "T", nullable={"qty"}, name="ok").filter(col("qty").gt(lit(1))).aggregate(
        [], [("count", star())])
    _lib.Module(_lib.codegen(plan.text()), key="plain_names_compile")
