"""Writes pwdft_api.json for the static check of the Julia binding
(tests/test_julia_shim.py), read as text from PWDFT.jl's src/:

  structs    fields (name and declared type) of Hamiltonian, PsPot_GTH and
             every struct reachable from them through field types
  functions  for each PWDFT.<name> the binding uses, and for the drivers it
             documents, whether src/ defines a function of that name
  methods    for each function the binding adds methods to, the positional
             parameter types of every method src/ defines for it ("Any" where
             untyped): what the binding's invoke calls must name
  gth_typed  the functions src/ defines with a parameter typed
             Hamiltonian{PsPot_GTH}, PsPot_GTH or Vector{PsPot_GTH}: none of
             them takes the binding's Hamiltonian{PsPot_GTH_B200} or its
             species, so the binding must add a method for each
  calls      every call in src/ of a function the binding adds methods to:
             file:line, the kind of each positional argument ("bloch": a
             whole BlochWavefunc such as psiks, "block": an indexed one such
             as psiks[ik], "splat", or "unknown") and the keyword names (what
             PWDFT's own drivers pass to the binding's methods)

Run where the reference sources are present:

    python tests/golden/make_pwdft_api.py <PWDFT.jl checkout>/src

Julia syntax handled: `[mutable] struct Name{params} [<: Super]` blocks whose
fields are `name::Type` or bare `name` lines at the block's own depth (inner
constructors are skipped), `abstract type Name ... end`, `function name(`
definitions and one-line `name(args) = ...` methods (an optional module
prefix such as `Base.` is dropped).
"""
import json
import os
import re
import sys

BLOCK_OPEN = re.compile(r"^\s*(function|if|for|while|let|begin|do|quote|try|macro|module|struct|mutable\s+struct)\b")
BLOCK_OPEN_INLINE = re.compile(r"\bdo\b(\s+\w+(\s*,\s*\w+)*)?\s*$")
END = re.compile(r"^\s*end\b")
STRUCT = re.compile(r"^\s*(?:mutable\s+)?struct\s+([A-Za-z_]\w*)")
FIELD = re.compile(r"^\s*([A-Za-z_]\w*)\s*(?:::\s*(.+?))?\s*(?:#.*)?$")
FUNC = re.compile(r"^\s*function\s+(?:[A-Za-z_]\w*\.)?([A-Za-z_][\w!]*)\s*[({]")
ONELINER = re.compile(r"^(?:[A-Za-z_]\w*\.)?([A-Za-z_][\w!]*)\s*(?:\{[^}]*\})?\s*\(.*\)\s*(?:where\s*\{?[^=]*\}?)?\s*=[^=]")
ABSTRACT = re.compile(r"^\s*abstract\s+type\s+([A-Za-z_]\w*)")
KEYWORDS = {"end", "function", "if", "else", "elseif", "for", "while", "return", "begin", "let", "local", "global",
            "const", "using", "import", "export", "include", "try", "catch", "finally"}


def strip_strings(line):
    return re.sub(r'"(?:[^"\\]|\\.)*"', '""', line)


def parse_file(path, structs, functions, abstract):
    with open(path, encoding="utf-8", errors="replace") as f:
        lines = f.read().split("\n")
    i = 0
    in_doc = False
    while i < len(lines):
        raw = lines[i]
        if raw.strip().startswith('"""'):
            # docstring block: skip to its closing quotes
            if not (raw.strip().count('"""') >= 2 and len(raw.strip()) > 3):
                in_doc = not in_doc
            i += 1
            continue
        if in_doc:
            i += 1
            continue
        line = strip_strings(raw)
        m = ABSTRACT.match(line)
        if m:
            abstract.add(m.group(1))
        m = FUNC.match(line)
        if m:
            functions.add(m.group(1))
        m = ONELINER.match(line)
        if m and m.group(1) not in KEYWORDS:
            functions.add(m.group(1))
        m = STRUCT.match(line)
        if m:
            name = m.group(1)
            fields = []
            depth = 1
            i += 1
            while i < len(lines) and depth > 0:
                body = strip_strings(lines[i]).split("#")[0]
                if END.match(body):
                    depth -= 1
                elif BLOCK_OPEN.match(body) or BLOCK_OPEN_INLINE.search(body):
                    if depth == 1:
                        fm = FUNC.match(body)
                        if fm:
                            functions.add(fm.group(1))
                    depth += 1
                elif depth == 1:
                    fm = FIELD.match(body)
                    if fm and fm.group(1) not in KEYWORDS and body.strip():
                        fields.append([fm.group(1), (fm.group(2) or "Any").strip()])
                i += 1
            structs[name] = fields
            continue
        i += 1


SHIM = os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
                    "pwdft.jl_b200", "julia", "PWDFTB200.jl")
DRIVERS = ["KS_solve_SCF!", "KS_solve_Emin_PCG!", "diag_davidson!", "diag_Emin_PCG!", "diag_CheFSI!"]


def julia_code(text):
    """Julia source without docstrings, string literals and comments (line
    numbers kept)."""
    text = re.sub(r'"""(?:.|\n)*?"""', lambda m: '""' + "\n" * m.group(0).count("\n"), text)
    text = re.sub(r'"(?:[^"\\\n]|\\.)*"', '""', text)
    return re.sub(r"#.*", "", text)


def split_top(args):
    """Top-level comma split of an argument list (nesting by ()[]{})."""
    out, depth, cur = [], 0, ""
    for ch in args:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def call_sites(code, name):
    """(line, positional expressions, keyword names) of each call of name."""
    sites = []
    for m in re.finditer(r"(?<![\w.!])(?:PWDFT\.)?" + re.escape(name) + r"\(", code):
        start = m.end()
        before = code[:m.start()]
        line_start = before.rfind("\n") + 1
        prefix = code[line_start:m.start()]
        if re.search(r"\bfunction\s*$", prefix):
            continue                       # a definition
        depth, j = 1, start
        while j < len(code) and depth:
            depth += {"(": 1, ")": -1}.get(code[j], 0)
            j += 1
        inner = code[start:j - 1]
        if re.match(r"\s*=[^=]", code[j:j + 3]) and not prefix.strip():
            continue                       # a one-line method definition
        pos_part, _, kw_part = inner.partition(";")
        pos, kws = [], []
        for a in split_top(pos_part):
            a = " ".join(a.split())
            km = re.match(r"^([A-Za-z_]\w*)\s*=(?!=)", a)
            if km:
                kws.append(km.group(1))
            elif a:
                pos.append(a)
        for a in split_top(kw_part):
            km = re.match(r"^([A-Za-z_]\w*)\s*(?:=(?!=)|$)", " ".join(a.split()))
            if km:
                kws.append(km.group(1))
        sites.append((before.count("\n") + 1, pos, sorted(kws)))
    return sites


def method_signatures(code, name):
    """Positional parameter types of each `function name(...)` in code."""
    sigs = []
    for m in re.finditer(r"^\s*function\s+(?:PWDFT\.)?" + re.escape(name) + r"\s*\(", code, re.M):
        depth, j = 1, m.end()
        while j < len(code) and depth:
            depth += {"(": 1, ")": -1}.get(code[j], 0)
            j += 1
        pos = code[m.end():j - 1].partition(";")[0]
        types = []
        for a in split_top(pos):
            a = " ".join(a.split())
            if not a:
                continue
            tm = re.match(r"^\w+\s*::\s*(.+?)(?:\s*=.*)?$", a)
            types.append(tm.group(1).replace(" ", "") if tm else "Any")
        sigs.append(types)
    return sigs


GTH_TYPE = re.compile(r"::\s*(?:Hamiltonian\{PsPot_GTH\}|PsPot_GTH|Vector\{PsPot_GTH\}|Array\{PsPot_GTH,\s*1\})\s*(?:[,;=]|$)")


def gth_typed(code):
    """Names of the functions whose parameters include a GTH-typed one."""
    out = set()
    for m in re.finditer(r"^\s*function\s+(?:\w+\.)?([A-Za-z_][\w!]*)\s*\(", code, re.M):
        depth, j = 1, m.end()
        while j < len(code) and depth:
            depth += {"(": 1, ")": -1}.get(code[j], 0)
            j += 1
        if any(GTH_TYPE.search(" ".join(a.split())) for a in split_top(code[m.end():j - 1].replace(";", ","))):
            out.add(m.group(1))
    return out


def arg_kind(expr):
    if "..." in expr:
        return "splat"
    if expr.endswith("]"):
        return "block"
    if expr in ("psiks", "psic", "Hpsiks"):
        return "bloch"
    return "unknown"


def reachable(structs, roots):
    seen, todo = set(), list(roots)
    while todo:
        t = todo.pop()
        if t in seen or t not in structs:
            continue
        seen.add(t)
        for _, ty in structs[t]:
            todo.extend(re.findall(r"[A-Za-z_]\w*", ty))
    return seen


def main(src):
    structs, functions, abstract = {}, set(), set()
    for root, _, files in os.walk(src):
        for fn in sorted(files):
            if fn.endswith(".jl"):
                parse_file(os.path.join(root, fn), structs, functions, abstract)
    with open(SHIM) as f:
        code = julia_code(f.read())
    used = sorted(set(re.findall(r"\bPWDFT\.([A-Za-z_][\w!]*)", code)) | set(DRIVERS))
    keep = reachable(structs, ["Hamiltonian", "PsPot_GTH"])
    extended = sorted(set(re.findall(r"^(?:function\s+)?PWDFT\.([A-Za-z_][\w!]*)\(", code, re.M)))
    calls = {n: [] for n in extended}
    methods = {n: [] for n in extended}
    typed = set()
    for root, _, files in os.walk(src):
        for fn in sorted(files):
            if fn.endswith(".jl"):
                with open(os.path.join(root, fn), encoding="utf-8", errors="replace") as f:
                    ref = julia_code(f.read())
                rel = os.path.relpath(os.path.join(root, fn), os.path.dirname(src.rstrip("/")))
                typed |= gth_typed(ref)
                for n in extended:
                    methods[n] += method_signatures(ref, n)
                    for line, pos, kws in call_sites(ref, n):
                        calls[n].append({"at": "%s:%d" % (rel, line), "positional": [arg_kind(a) for a in pos],
                                         "keywords": kws})
    out = {"structs": {k: structs[k] for k in sorted(keep)},
           "functions": {n: n in functions for n in used if n not in abstract},
           "abstract_types": {n: True for n in used if n in abstract},
           "methods": methods,
           "gth_typed": sorted(typed),
           "calls": calls}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pwdft_api.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote", dst, len(out["structs"]), "structs", len(out["functions"]), "functions")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "src")
