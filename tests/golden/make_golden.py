"""Generate the golden fixtures that pin the CPU oracle to the reference's own code.

Runs the reference's standalone CPU engine (src/cpu/ssb/q11.cpp, q21.cpp, q41.cpp,
built unmodified under oracle/_ref by oracle/Makefile) on seeded synthetic tables and
records what it prints. The fixture stores the inputs' recipe (seed and sizes of the
generator in mordred_b200/csrc/ssbgen.h) and the outputs, so tests can regenerate the
inputs anywhere and compare the oracle (or the GPU) with the reference's answers.

The date table has the reference's 2,556 rows (no 19981231) and the reference's
61,130 date slots are kept, so fact rows dated 19981231 wrap onto 19920101's slot
exactly as in the reference.

usage: python tests/golden/make_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

CASES = [
    # seed, lo_len, s_len, c_len, p_len, d_len
    (1, 1000, 100, 300, 200, 2556),
    (7, 200_000, 2_000, 30_000, 20_000, 2556),
    (42, 1_000_003, 4_000, 60_000, 100_000, 2556),
]


def main():
    O.build_lib()
    out = []
    for seed, lo, s, c, p, d in CASES:
        case = {"seed": seed, "lo_len": lo, "s_len": s, "c_len": c, "p_len": p, "d_len": d,
                "d_val_len": 19981230 - 19920101 + 1}
        lines, _ = O.run_ref(11, seed, lo, s, c, p, d, threads=4)
        case["q11_revenue"] = O.parse_ref_revenue(lines)[-1]
        lines, _ = O.run_ref(21, seed, lo, s, c, p, d, threads=4)
        case["q21_groups"] = O.parse_ref_groups(lines)
        lines, _ = O.run_ref(41, seed, lo, s, c, p, d, threads=4)
        case["q41_groups"] = O.parse_ref_groups(lines)
        out.append(case)
        print(f"seed {seed}: q11 {case['q11_revenue']}, q21 {len(case['q21_groups'])} groups, "
              f"q41 {len(case['q41_groups'])} groups")
    with open(os.path.join(HERE, "reference_ssb.json"), "w") as f:
        json.dump({"generator": "mordred_b200/csrc/ssbgen.h", "source": "oracle/_ref (src/cpu/ssb)",
                   "cases": out}, f, indent=0)


if __name__ == "__main__":
    main()
