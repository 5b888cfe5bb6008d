"""Writes tests/golden/csv_ref.npz from the reference's own CSV reader:
csv-parser (the reference's vendored header) + std::stoi / std::stof /
strptime+timegm, replayed by oracle/csv_ref_harness.cpp and built into
oracle/_ref/libcsvref.so by `make -C oracle csvref` (CPU only). Inputs are the
seeded cases of tests/csv_cases.py; tests/test_csv_cpu.py checks the oracle
against the stored outputs.

    python tests/golden/make_csv_golden.py [--out DIR]
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from tests import csv_cases  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    rng = np.random.default_rng(2024)
    cases = csv_cases.edge_cases() + [csv_cases.random_csv(rng, max_rows=40) for _ in range(40)]
    arrays = {"count": np.array(len(cases))}
    for i, (types, header, body) in enumerate(cases):
        r = oracle.ref_csv_scan(header, body, types)
        arrays[f"body{i}"] = np.frombuffer(body, dtype=np.uint8) if body else np.zeros(0, np.uint8)
        arrays[f"types{i}"] = np.array(types, dtype=np.int32)
        arrays[f"meta{i}"] = np.array([r["rows"], r["bad"], r["first_row"], r["first_field"], r["first_kind"]],
                                      dtype=np.int64)
        for f, t in enumerate(types):
            if t >= 0:
                arrays[f"vals{i}_{f}"] = r["cols"][f][0]
                arrays[f"nulls{i}_{f}"] = r["cols"][f][1]
    np.savez_compressed(os.path.join(args.out, "csv_ref.npz"), **arrays)
    print("wrote", len(cases), "cases")


if __name__ == "__main__":
    main()
