"""Writes reference_line_counts.json: the number of lines of every .jl file
of the PWDFT.jl tree, keyed by file name (names that occur more than once
map to the largest count), for tests/test_citations.py.

Run where the reference sources are present:

    python tests/golden/make_line_counts.py <PWDFT.jl checkout>
"""
import json
import os
import sys


def main(top):
    counts = {}
    for root, _, files in os.walk(top):
        for fn in files:
            if fn.endswith(".jl"):
                with open(os.path.join(root, fn), encoding="utf-8", errors="replace") as f:
                    n = sum(1 for _ in f)
                counts[fn] = max(n, counts.get(fn, 0))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_line_counts.json")
    with open(dst, "w") as f:
        json.dump(dict(sorted(counts.items())), f, indent=0, sort_keys=True)
        f.write("\n")
    print("wrote", dst, len(counts), "files")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else ".")
