"""Static checks of the Julia binding (pwdft.jl_b200/julia/PWDFTB200.jl)
against PWDFT.jl's own types and call sites.  Julia is not installed here,
so the binding is checked as text against tests/golden/pwdft_api.json (made
by tests/golden/make_pwdft_api.py from the reference sources):

  constructor  on_device builds Hamiltonian{PsPot_GTH_B200} from Ham's
               fields in their declared order (pspots replaced)
  fields       every field chain on the Hamiltonian (Ham.pw.gvecw.kpoints.wk,
               Ham.pspots[i].psp.lmax, ...), on typed arguments and on the
               local names bound to such chains resolves through the declared
               field types
  names        every PWDFT.<name> the binding extends or calls, and every
               driver it documents, is defined by PWDFT.jl
  GTH methods  every function PWDFT.jl types on Hamiltonian{PsPot_GTH},
               PsPot_GTH or Vector{PsPot_GTH} (none accepts the binding's
               Hamiltonian{PsPot_GTH_B200} or its species) gets a method from
               the binding
  dispatch     every call in PWDFT.jl of a function the binding adds methods
               to, whose arguments fit one of those methods (by count and,
               where the argument shows it, whole BlochWavefunc vs one
               k-point's block), passes only keywords that method accepts; the
               drivers' own calls of diag_LOBPCG!, calc_rhoe!, update! and
               calc_grad reach the binding's methods
"""
import json
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "pwdft.jl_b200", "julia", "PWDFTB200.jl")
API = os.path.join(ROOT, "tests", "golden", "pwdft_api.json")


def julia_code(text):
    """Julia source without docstrings, string literals and comments (line
    numbers kept)."""
    text = re.sub(r'"""(?:.|\n)*?"""', lambda m: '""' + "\n" * m.group(0).count("\n"), text)
    text = re.sub(r'"(?:[^"\\\n]|\\.)*"', '""', text)
    return re.sub(r"#.*", "", text)


def split_top(args):
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


def balanced(code, start):
    """Text from code[start] (just after an opening parenthesis) to its
    matching closing parenthesis, exclusive, and the index after it."""
    depth, j = 1, start
    while j < len(code) and depth:
        depth += {"(": 1, ")": -1}.get(code[j], 0)
        j += 1
    return code[start:j - 1], j


def load():
    with open(API) as f:
        api = json.load(f)
    with open(SHIM) as f:
        code = julia_code(f.read())
    return api, code


def shim_structs(code):
    out = {}
    for m in re.finditer(r"^(?:mutable\s+)?struct\s+(\w+)[^\n]*\n((?:(?!^end\b).*\n)*?)^end\b", code, re.M):
        out[m.group(1)] = [list(f) for f in re.findall(r"^\s*(\w+)::(\S+)", m.group(2), re.M)]
    return out


class Types:
    def __init__(self, api, code):
        self.s = dict(api["structs"])
        self.s.update(shim_structs(code))

    def field(self, t, f):
        for name, ty in self.s.get(t, []):
            if name == f:
                return ty.replace("Tpsp", "PsPot_GTH_B200")
        if t == "PsPot_GTH_B200":       # Base.getproperty forwards to the GTH record
            return self.field("PsPot_GTH", f)
        return None

    def structs_in(self, ty):
        return [w for w in re.findall(r"[A-Za-z_]\w*", ty) if w in self.s]


def chains(expr):
    """(root, [fields]) of every dotted chain in expr, index expressions
    scanned on their own."""
    pieces, todo = [], [expr]
    while todo:
        e = todo.pop()
        while True:
            m = re.search(r"\[([^\[\]]*)\]", e)
            if not m:
                break
            todo.append(m.group(1))
            e = e[:m.start()] + "\x00" + e[m.end():]
        pieces.append(e)
    out = []
    for e in pieces:
        for m in re.finditer(r"(?<![\w.])([A-Za-z_]\w*)((?:\x00?\.[A-Za-z_]\w*)+)", e):
            out.append((m.group(1), re.findall(r"\.([A-Za-z_]\w*)", m.group(2))))
    return out


def resolve(types, start, fields):
    """Types reached by following fields from the candidate types start;
    raises AssertionError naming the first field no candidate declares."""
    cur = list(start)
    for i, f in enumerate(fields):
        nxt, found = [], False
        for t in cur:
            ft = types.field(t, f)
            if ft is not None:
                found = True
                nxt += types.structs_in(ft)
        assert found, "no field %r in %s" % (f, cur)
        if not nxt and i + 1 < len(fields):
            raise AssertionError("field access after %r, which is not a struct" % f)
        cur = nxt
    return cur


def top_level_blocks(code):
    """(first line, text) of each top-level definition of the module."""
    lines = code.split("\n")
    starts = [i for i, l in enumerate(lines)
              if re.match(r"^(function\s|[A-Za-z_][\w.!]*(\{[^}]*\})?\(.*\)\s*=|[A-Za-z_][\w.!]*\(.*\)\s*=\s*$)", l)]
    starts.append(len(lines))
    return [(a + 1, "\n".join(lines[a:b])) for a, b in zip(starts, starts[1:])]


def test_constructor_matches_hamiltonian_fields():
    api, code = load()
    m = re.search(r"Hamiltonian\{PsPot_GTH_B200\}\(", code)
    assert m, "on_device does not build a Hamiltonian{PsPot_GTH_B200}"
    args, _ = balanced(code, m.end())
    args = [" ".join(a.split()) for a in split_top(args)]
    fields = [f for f, _ in api["structs"]["Hamiltonian"]]
    assert len(args) == len(fields), (args, fields)
    for a, f in zip(args, fields):
        assert a == ("pspots" if f == "pspots" else "Ham." + f), (a, f)


def test_field_chains_resolve():
    api, code = load()
    types = Types(api, code)
    checked = 0
    for line0, block in top_level_blocks(code):
        sig = re.match(r"^(?:function\s+)?[\w.!]+(?:\{[^}]*\})?\(", block)
        env = {}
        if sig:
            params, _ = balanced(block, sig.end())
            for p in split_top(params.replace(";", ",")):
                pm = re.match(r"^(\w+)::(.+?)(?:=.*)?$", p.strip())
                if pm:
                    ty = pm.group(2).strip()
                    if ty in ("B200Hamiltonian", "Hamiltonian{PsPot_GTH}") or ty.startswith("Hamiltonian"):
                        env[pm.group(1)] = ["Hamiltonian"]
                    elif ty in types.s:
                        env[pm.group(1)] = [ty]
        for k, line in enumerate(block.split("\n")):
            am = re.match(r"^\s*(\w+)\s*=\s*([A-Za-z_][\w.\[\]+\-* ]*?)\s*$", line)
            for root, fields in chains(line):
                if root in env:
                    try:
                        resolve(types, env[root], fields)
                    except AssertionError as e:
                        raise AssertionError("PWDFTB200.jl:%d: %s.%s: %s" % (line0 + k, root, ".".join(fields), e))
                    checked += 1
            if am:
                cs = chains(am.group(2))
                whole = am.group(2)
                while re.search(r"\[[^\[\]]*\]", whole):
                    whole = re.sub(r"\[[^\[\]]*\]", "", whole)
                whole = whole.replace(" ", "")
                bound = [c for c in cs if c[0] in env and whole == c[0] + "." + ".".join(c[1])]
                if bound:
                    env[am.group(1)] = resolve(types, env[bound[0][0]], bound[0][1])
    assert checked > 60, checked


def test_pwdft_names_exist():
    api, code = load()
    used = set(re.findall(r"\bPWDFT\.([A-Za-z_][\w!]*)", code))
    assert used, "the binding names no PWDFT function"
    for n in sorted(used):
        assert api["functions"].get(n) or api["abstract_types"].get(n), "PWDFT.%s is not defined by PWDFT.jl" % n
    for n in ("KS_solve_SCF!", "KS_solve_Emin_PCG!", "diag_davidson!", "diag_Emin_PCG!", "diag_CheFSI!"):
        assert api["functions"][n], n


def shim_methods(code):
    """name -> [(positional (name, kind) list, keyword names, takes kwargs...)]"""
    out = {}
    for m in re.finditer(r"^(?:function\s+)?PWDFT\.([A-Za-z_][\w!]*)\(", code, re.M):
        params, _ = balanced(code, m.end())
        pos_part, _, kw_part = params.partition(";")
        pos = []
        for p in split_top(pos_part):
            pm = re.match(r"^(\w+)(?:::(.+))?$", " ".join(p.split()))
            ty = (pm.group(2) or "") if pm else ""
            kind = ("bloch" if "BlochWavefunc" in ty else
                    "array" if re.search(r"Matrix|Array|VecOrMat|Vector", ty) else "any")
            pos.append((p, kind))
        kws = [re.match(r"\s*(\w+)", k).group(1) for k in split_top(kw_part)]
        out.setdefault(m.group(1), []).append((pos, kws, any(k.endswith("...") for k in split_top(kw_part))))
    return out


def fits(method_pos, kinds):
    """Whether a call with argument kinds (bloch / block / splat / unknown)
    can dispatch to a method with these positional parameters."""
    if any("..." in p for p, _ in method_pos) or "splat" in kinds:
        return False
    if len(method_pos) != len(kinds):
        return False
    for (_, pk), ak in zip(method_pos, kinds):
        if ak == "bloch" and pk == "array" or ak == "block" and pk == "bloch":
            return False
    return True


def test_driver_calls_dispatch_with_accepted_keywords():
    api, code = load()
    methods = shim_methods(code)
    reached = set()
    for name, sites in api["calls"].items():
        assert name in methods, name
        for site in sites:
            fit = [m for m in methods[name] if fits(m[0], site["positional"])]
            if not fit:
                continue                  # PWDFT's own method takes this call
            if any(m[2] for m in fit):
                continue
            accepted = set().union(*[set(m[1]) for m in fit])
            missing = set(site["keywords"]) - accepted
            assert not missing, "%s calls %s with keywords %s the binding's method does not take" % (
                site["at"], name, sorted(missing))
            reached.add((site["at"].split(":")[0], name))
    for f, n in (("src/KS_solve_SCF.jl", "diag_LOBPCG!"), ("src/KS_solve_SCF.jl", "calc_rhoe!"),
                 ("src/KS_solve_SCF.jl", "update!"), ("src/KS_solve_Emin_PCG.jl", "calc_grad"),
                 ("src/KS_solve_Emin_PCG.jl", "calc_rhoe!")):
        assert (f, n) in reached, (f, n)


def test_every_gth_typed_method_is_covered():
    api, code = load()
    extended = set(re.findall(r"^(?:function\s+)?PWDFT\.([A-Za-z_][\w!]*)(?:\{[^}]*\})?\(", code, re.M))
    missing = sorted(set(api["gth_typed"]) - extended)
    assert not missing, "PWDFT methods typed on the GTH types with no method for the binding's types: %s" % missing
