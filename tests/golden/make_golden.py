"""Extracts the reference's known-answer vectors for the hot path into
tests/golden/reference_kats.json (run here, where the reference is mounted;
the JSON travels with the repository).

Sources (paths inside the reference project, read as text):
  test/nullable_data/nullable_numbers.csv, queries.sql, expected.tsv
      12-row nullable table and the expected outputs of q1-q5;
  test/test_sql_3vl.cpp:91-99
      SQL three-valued-logic truth-table assertions;
  test/test_nullable_semantics.cpp:13-57
      validity-bitmap decoding cases (valid8 / null8 / null64);
  test/test_optimizer.cpp:280,305,394
      result-size known answers (Q2.1 shape 21000, scalar 1, Q3.1 shape 17500).

Usage: python tests/golden/make_golden.py [/path/to/reference]
"""
from __future__ import annotations

import csv
import json
import os
import re
import sys
from pathlib import Path

REF = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CRYSTAL_REFERENCE", "/root/reference"))
OUT = Path(__file__).resolve().parent / "reference_kats.json"


def nullable_kat() -> dict:
    d = REF / "test" / "nullable_data"
    with open(d / "nullable_numbers.csv") as f:
        rows = list(csv.DictReader(f))
    cols = list(rows[0].keys())
    table = {c: [int(r[c]) if r[c] != "" else None for r in rows] for c in cols}
    expected: dict[str, dict] = {}
    for line in (d / "expected.tsv").read_text().splitlines():
        parts = line.split("\t")
        q, vals = parts[0], parts[1:]
        if q not in expected:
            expected[q] = {"columns": vals, "rows": []}
        else:
            expected[q]["rows"].append([float(v) if "." in v else int(v) for v in vals])
    queries = {}
    cur = None
    for line in (d / "queries.sql").read_text().splitlines():
        m = re.match(r"--\s*(q\d+)", line)
        if m:
            cur = m.group(1)
            queries[cur] = ""
        elif cur and line.strip():
            queries[cur] += line.strip() + " "
    return {"columns": table, "expected": expected, "queries": {k: v.strip() for k, v in queries.items()}}


def truth_table() -> list[dict]:
    src = (REF / "test" / "test_sql_3vl.cpp").read_text()
    out = []
    for fn, a, b, r in re.findall(r"assert\(sql_(and|or)\(SqlBool::(\w+), SqlBool::(\w+)\) == SqlBool::(\w+)\)", src):
        out.append({"op": fn, "a": a, "b": b, "result": r})
    for a, r in re.findall(r"assert\(sql_not\(SqlBool::(\w+)\) == SqlBool::(\w+)\)", src):
        out.append({"op": "not", "a": a, "result": r})
    return out


def bitmap_cases() -> list[dict]:
    src = (REF / "test" / "test_nullable_semantics.cpp").read_text()
    cases = []
    for m in re.finditer(r"static void (test_\w+)\(\) \{(.*?)\n\}", src, re.S):
        name, body = m.group(1), m.group(2)
        bytes_m = re.search(r"std::vector<unsigned char> bytes = \{([^}]*)\}", body)
        words_m = re.search(r"std::vector<uint64_t> null_words = \{0b([01]+)ULL\}", body)
        call = re.search(r"decodeValidity(Byte|Word)Bitmap\([^,]+,\s*(\w+(?:\.size\(\))?|\d+),\s*(true|false)\)", body)
        checks = [(bool(neg == ""), int(row)) for neg, row in re.findall(r"assert\((!?)bit_at\(validity, (\d+)\)\)", body)]
        throws = "thrown" in body
        if not call:
            continue
        case = {"name": name, "kind": call.group(1).lower(), "input_is_valid": call.group(3) == "true",
                "expect": [[row, valid] for valid, row in checks], "throws": throws}
        if bytes_m:
            case["bytes"] = [int(x) for x in bytes_m.group(1).split(",")]
        if words_m:
            case["word"] = int(words_m.group(1), 2)
        rows_arg = call.group(2)
        case["rows"] = len(case.get("bytes", [])) if rows_arg.endswith(".size()") else int(rows_arg)
        cases.append(case)
    bad = re.search(r"decodeValidityByteBitmap\(std::vector<unsigned char>\{([^}]*)\}, (\d+), (true|false)\)", src)
    if bad:
        cases.append({"name": "test_invalid_byte_count_throws", "kind": "byte",
                      "bytes": [int(x) for x in bad.group(1).split(",")], "rows": int(bad.group(2)),
                      "input_is_valid": bad.group(3) == "true", "expect": [], "throws": True})
    return cases


def result_sizes() -> list[dict]:
    src = (REF / "test" / "test_optimizer.cpp").read_text()
    out = []
    for size, msg in re.findall(r"assert\(size == (\d+) && \"([^\"]+)\"\)", src):
        out.append({"size": int(size), "what": msg})
    return out


def main() -> None:
    data = {
        "source": "aidarxa/practice test fixtures (see make_golden.py for file list)",
        "nullable_kat": nullable_kat(),
        "sql_3vl": truth_table(),
        "validity_decode": bitmap_cases(),
        "result_sizes": result_sizes(),
    }
    OUT.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
