"""The Lisp binding (lisp/fmgpu.lisp) cannot be loaded here (no Common Lisp
implementation), so its consistency with the C-ABI and with Femlisp is
checked by reading it:

* the file is balanced s-expressions;
* every fl.port:def-function binds a function the header declares, with the
  header's number of arguments, and every argument and return type is one
  that fl.port:convert-type (src/basic/port.lisp:381-398) maps or passes
  through to SBCL's define-alien-routine, matching the C parameter type
  (handles as integers, T** handles as (* sb-alien:unsigned-long), struct
  pointers and C strings as octet vectors);
* every package-qualified symbol exists: fl.* symbols with one colon are
  exported by the reference's defpackage forms, with two colons exported,
  a class of that package or a slot name of one (tests/golden/femlisp_exports.json,
  made by tests/golden/make_femlisp_exports.py); sb-alien / sb-sys symbols
  are SBCL exports the binding needs;
* the drop-in classes carry their methods: make-iterator for
  <gpu-geometric-cs> and <gpu-cg>, solve for <gpu-linear-solver>, the device
  hierarchy for <gpu-geometric-cs> (structured) and <gpu-local-mg>
  (algebraic, for locally refined meshes).
"""
import json
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LISP = os.path.join(ROOT, "lisp", "fmgpu.lisp")

# types convert-type maps for SBCL (port.lisp:381-398) and the SB-ALIEN type
# names the binding passes through it
MAPPED = {":void", ":char", ":int", ":float", ":double"}
SB_ALIEN_TYPES = {"sb-alien:long", "sb-alien:unsigned-long"}
SBCL_SYMBOLS = SB_ALIEN_TYPES | {"sb-sys:with-pinned-objects", "sb-sys:vector-sap", "sb-sys:sap-ref-32",
                                 "sb-sys:sap-ref-double"}
HANDLES = {"fmg_ctx", "fmg_grid", "fmg_vec", "fmg_net"}


def _tokens(text):
    i, n = 0, len(text)
    while i < n:
        c = text[i]
        if c == ";":
            while i < n and text[i] != "\n":
                i += 1
        elif c == '"':
            j = i + 1
            while j < n and text[j] != '"':
                j += 2 if text[j] == "\\" else 1
            yield ("str", text[i + 1:j])
            i = j + 1
        elif c in "()":
            yield (c, c)
            i += 1
        elif c.isspace() or c in "'`,":
            i += 1
        else:
            j = i
            while j < n and not text[j].isspace() and text[j] not in '()";':
                j += 1
            yield ("atom", text[i:j])
            i = j


class LStr(str):
    """A Lisp string literal (kept apart from symbols)."""


def _read(text):
    stack, top = [], []
    for kind, val in _tokens(text):
        if kind == "str":
            top.append(LStr(val))
            continue
        if kind == "(":
            stack.append(top)
            top = []
        elif kind == ")":
            assert stack, "unbalanced ')'"
            done = top
            top = stack.pop()
            top.append(done)
        else:
            top.append(val)
    assert not stack, "unbalanced '('"
    return top


def _forms():
    return _read(open(LISP).read())


def _header():
    h = open(os.path.join(ROOT, "include", "fmgpu.h")).read()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(int|long|void)\s+(fmg_\w+)\s*\(([^)]*)\)\s*;", h):
        params = [a.strip() for a in m.group(3).split(",") if a.strip() and a.strip() != "void"]
        types = []
        for p in params:
            p = re.sub(r"\bconst\b", "", p)
            p = re.sub(r"\s+", " ", p).strip()
            t = re.sub(r"\s*\b\w+$", "", p).replace(" *", "*").strip()
            types.append(t)
        out[m.group(2)] = (m.group(1), types)
    return out


def _lisp_type(t):
    return t if isinstance(t, str) else "(" + " ".join(_lisp_type(x) for x in t) + ")"


def _expected(ctype):
    """The binding's type for a C parameter type."""
    stars = ctype.count("*")
    base = ctype.replace("*", "").strip()
    if base in HANDLES:
        return {1: "sb-alien:unsigned-long", 2: "(* sb-alien:unsigned-long)"}[stars]
    if base in ("fmg_solve_cfg", "fmg_mixed_cfg", "char"):
        return "(* :char)"
    scalar = {"int": ":int", "long": "sb-alien:long", "double": ":double", "float": ":float"}[base]
    return scalar if stars == 0 else "(* " + scalar + ")"


def _accepted(t):
    if isinstance(t, str):
        return t in MAPPED or t in SB_ALIEN_TYPES
    return len(t) == 2 and t[0] == "*" and _accepted(t[1])


def _def_functions():
    return [f for f in _forms() if isinstance(f, list) and f and f[0] == "fl.port:def-function"]


def test_lisp_binding_matches_the_header():
    hdr = _header()
    bound = _def_functions()
    assert len(bound) >= 15
    for f in bound:
        cname, args = f[1][0], f[2]
        assert cname in hdr, f"{cname} is not declared in include/fmgpu.h"
        ret, ctypes_ = hdr[cname]
        assert len(args) == len(ctypes_), f"{cname}: {len(args)} arguments bound, header has {len(ctypes_)}"
        kw = dict(zip(f[3::2], f[4::2]))
        assert kw.get(":returning") == (":int" if ret == "int" else "sb-alien:long"), (cname, kw)
        for (name, t), ct in zip(args, ctypes_):
            assert _accepted(t), f"{cname} {name}: type {_lisp_type(t)} is not one convert-type hands to SBCL"
            assert _lisp_type(t) == _expected(ct), f"{cname} {name}: {_lisp_type(t)} for C type {ct}"


def _symbols(form, out):
    if isinstance(form, list):
        for x in form:
            _symbols(x, out)
    elif isinstance(form, str) and not isinstance(form, LStr) and re.match(r"^[a-z][\w.\-]*::?[^:]", form, re.I) and not form.startswith("#"):
        out.add(form)


def test_package_qualified_symbols_exist():
    table = json.load(open(os.path.join(ROOT, "tests", "golden", "femlisp_exports.json")))
    names = {}
    for p, v in table.items():
        names[p] = v
        for nick in v["nicknames"]:
            names[nick] = v
    syms = set()
    _symbols(_forms(), syms)
    assert syms
    for s in sorted(syms):
        low = s.lower()
        if low.startswith(("sb-alien:", "sb-sys:")):
            assert low in SBCL_SYMBOLS, f"{s}: not among the SBCL symbols the binding may use"
            continue
        internal = "::" in s
        pkg, sym = re.split(r"::?", s, maxsplit=1)
        pkg, sym = pkg.upper(), sym.upper()
        assert pkg in names, f"{s}: package {pkg} is not defined by the reference"
        ok = sym in names[pkg]["exports"] or (internal and (sym in names[pkg].get("slots", [])
                                                            or sym in names[pkg].get("classes", [])))
        assert ok, f"{s}: not {'exported, a slot or a class' if internal else 'exported'} in {pkg}"
    assert not any(s.lower().startswith("fl.port:sap-ref") for s in syms)


def test_drop_in_classes_have_their_methods():
    forms = _forms()
    classes = {f[1]: f[2] for f in forms if isinstance(f, list) and f and f[0] == "defclass"}
    assert classes.get("<gpu-geometric-cs>") == ["fl.geomg:<geometric-cs>"]
    assert classes.get("<gpu-cg>") == ["fl.iteration:<cg>"]
    assert classes.get("<gpu-linear-solver>") == ["fl.iteration:<linear-solver>"]
    assert classes.get("<gpu-local-mg>") == ["<gpu-geometric-cs>", "fl.geomg::<local-mg>"]
    methods = {(f[1], f[2][0][1]) for f in forms if isinstance(f, list) and f and f[0] == "defmethod"}
    assert ("fl.iteration:make-iterator", "<gpu-geometric-cs>") in methods
    assert ("fl.iteration:make-iterator", "<gpu-cg>") in methods
    assert ("fl.iteration:solve", "<gpu-linear-solver>") in methods
    assert ("gpu-hierarchy", "<gpu-geometric-cs>") in methods
    assert ("gpu-hierarchy", "<gpu-local-mg>") in methods


def _struct_offsets(forms, defun_name):
    """Byte offsets of the fields of the (%struct size ...) form in the defun."""
    def find(form):
        if isinstance(form, list):
            if form and form[0] == "%struct":
                return form
            for x in form:
                got = find(x)
                if got is not None:
                    return got
        return None
    for f in forms:
        if isinstance(f, list) and len(f) > 1 and f[0] == "defun" and f[1] == defun_name:
            st = find(f)
            return int(st[1]), [int(fl[0]) for fl in st[2:] if isinstance(fl, list)]
    raise AssertionError(defun_name)


def test_config_struct_offsets_match_the_header():
    # fmg_solve_cfg / fmg_mixed_cfg as the binding lays them out (x86-64)
    import ctypes

    from gnu_femlisp_b200 import _capi as C
    forms = _forms()
    size, offs = _struct_offsets(forms, "%cfg-bytes")
    assert size == ctypes.sizeof(C.SolveCfg) == 72
    assert offs == [getattr(C.SolveCfg, f).offset for f, _ in C.SolveCfg._fields_]
    size, offs = _struct_offsets(forms, "%mixed-cfg-bytes")
    assert size == ctypes.sizeof(C.MixedCfg) == 24
    assert offs == [getattr(C.MixedCfg, f).offset for f, _ in C.MixedCfg._fields_]
