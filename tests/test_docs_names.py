"""The names the integration and design documents point a user at exist:
every `pwb200.<module>[.<name>]` resolves in the Python package, and every
`pw_<name>` C entry point is declared in include/pwb200.h (CPU only; nothing
is called).
"""
import importlib
import os
import re
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DOCS = ("INTEGRATION.md", "DESIGN.md", "README.md")


def _text():
    return "\n".join(open(os.path.join(ROOT, d), encoding="utf-8").read() for d in DOCS)


def test_python_names_resolve():
    sys.path.insert(0, os.path.join(ROOT, "pwdft.jl_b200"))
    names = sorted(set(re.findall(r"`(pwb200(?:\.[A-Za-z_]\w*)+)`", _text())))
    assert len(names) > 8, names
    for dotted in names:
        parts = dotted.split(".")
        obj, i = None, len(parts)
        while i > 0:                      # longest importable module prefix
            try:
                obj = importlib.import_module(".".join(parts[:i]))
                break
            except ImportError:
                i -= 1
        assert obj is not None, dotted
        for p in parts[i:]:
            assert hasattr(obj, p), dotted
            obj = getattr(obj, p)


def test_c_names_declared():
    header = open(os.path.join(ROOT, "include", "pwb200.h")).read()
    declared = set(re.findall(r"\b(pw_[a-z0-9_]+)\s*\(", header)) | set(re.findall(r"\b(pw_[a-z0-9_]+)\b", header))
    used = set(re.findall(r"`(pw_[a-z0-9_]+)(?=[(`])", _text()))   # calls, not file names
    missing = sorted(n for n in used if n not in declared)
    assert not missing, missing
