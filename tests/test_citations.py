"""Every reference citation `name.jl:a` or `name.jl:a-b` in this
repository's sources and documents names a file of the PWDFT.jl tree, with
1 <= a <= b <= the file's line count (tests/golden/reference_line_counts.json,
made by tests/golden/make_line_counts.py from the reference sources).
"""
import json
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COUNTS = os.path.join(ROOT, "tests", "golden", "reference_line_counts.json")
SKIP_DIRS = {".git", "_work", "gpurun_out", "baseline", "_build", "__pycache__", "golden"}
# documents written outside this repository's build (the survey, reviews and
# the baseline record) are not checked
SKIP_FILES = {"SURVEY.md", "VERDICT.md", "ADVICE.md", "BASELINE.md"}
EXT = (".h", ".c", ".cu", ".cuh", ".cpp", ".py", ".jl", ".md")
CITE = re.compile(r"\b([A-Za-z_][\w]*\.jl):(\d+)(?:-(\d+))?")


def sources():
    for root, dirs, files in os.walk(ROOT):
        dirs[:] = [d for d in dirs if d not in SKIP_DIRS]
        for fn in files:
            if fn.endswith(EXT) and fn not in SKIP_FILES and os.path.relpath(root, ROOT) != "tests/golden":
                yield os.path.join(root, fn)


def test_reference_citations_in_range():
    with open(COUNTS) as f:
        counts = json.load(f)
    bad, n = [], 0
    for path in sources():
        with open(path, encoding="utf-8", errors="replace") as f:
            text = f.read()
        for m in CITE.finditer(text):
            name, a = m.group(1), int(m.group(2))
            b = int(m.group(3) or a)
            n += 1
            rel = os.path.relpath(path, ROOT)
            if name not in counts:
                bad.append("%s: %s names no file of the reference" % (rel, m.group(0)))
            elif not 1 <= a <= b <= counts[name]:
                bad.append("%s: %s outside 1-%d" % (rel, m.group(0), counts[name]))
    assert n > 300, n
    assert not bad, "\n".join(bad)
