"""The Lisp binding (lisp/fmgpu.lisp) cannot be loaded here (no Common Lisp
implementation), so its consistency with the C-ABI is checked by reading it:
the file is balanced s-expressions, and every fl.port:def-function binds a
function the header declares, with the header's number of arguments."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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
        elif c.isspace():
            i += 1
        else:
            j = i
            while j < n and not text[j].isspace() and text[j] not in '()";':
                j += 1
            yield ("atom", text[i:j])
            i = j


def _read(text):
    stack, top = [], []
    for kind, val in _tokens(text):
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


def _header_arity():
    h = open(os.path.join(ROOT, "include", "fmgpu.h")).read()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(?:int|long|void)\s+(fmg_\w+)\s*\(([^)]*)\)\s*;", h):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = len(args)
    return out


def test_lisp_binding_matches_the_header():
    forms = _read(open(os.path.join(ROOT, "lisp", "fmgpu.lisp")).read())
    arity = _header_arity()
    bound = 0
    for f in forms:
        if isinstance(f, list) and f and f[0] == "fl.port:def-function":
            cname = f[1][0]
            assert cname in arity, f"{cname} is not declared in include/fmgpu.h"
            assert len(f[2]) == arity[cname], f"{cname}: {len(f[2])} arguments bound, header has {arity[cname]}"
            bound += 1
    assert bound >= 10
