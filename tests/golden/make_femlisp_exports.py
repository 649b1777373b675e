"""Writes femlisp_exports.json: for every package the reference's sources
define (defpackage), its names and nicknames, the symbol names it exports
and the names and slot names of the classes defined in it (defclass).  The Lisp binding's test checks every package-qualified symbol in
lisp/fmgpu.lisp against this table (no Lisp implementation runs here).

Run from the repository root with the reference checked out:
    python tests/golden/make_femlisp_exports.py /path/to/femlisp
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def tokens(text):
    i, n = 0, len(text)
    while i < n:
        c = text[i]
        if c == ";":
            while i < n and text[i] != "\n":
                i += 1
        elif c == "#" and i + 1 < n and text[i + 1] == "|":
            j = text.find("|#", i + 2)
            i = n if j < 0 else j + 2
        elif c == '"':
            j = i + 1
            while j < n and text[j] != '"':
                j += 2 if text[j] == "\\" else 1
            yield ("str", text[i + 1:j])
            i = j + 1
        elif c in "()":
            yield (c, c)
            i += 1
        elif c.isspace() or c == "'":
            i += 1
        else:
            j = i
            while j < n and not text[j].isspace() and text[j] not in '()";':
                j += 1
            yield ("atom", text[i:j])
            i = j


def read(text):
    stack, top = [], []
    for kind, val in tokens(text):
        if kind == "(":
            stack.append(top)
            top = []
        elif kind == ")":
            if not stack:
                continue
            done = top
            top = stack.pop()
            top.append(done)
        else:
            top.append(("s", val) if kind == "str" else val)
    return top


def name(x):
    if isinstance(x, tuple):
        return x[1].upper()
    s = str(x)
    for p in ("#:", ":"):
        if s.startswith(p):
            s = s[len(p):]
    return s.upper()


def main(root):
    pkgs = {}
    for dirpath, _, files in os.walk(os.path.join(root, "src")):
        for f in sorted(files):
            if not f.endswith(".lisp"):
                continue
            text = open(os.path.join(dirpath, f), encoding="utf-8", errors="replace").read()
            stack = read(text)
            # defclass slot names, by the package of the in-package form before them
            cur = None
            for form in stack:
                if not isinstance(form, list) or not form or not isinstance(form[0], str):
                    continue
                head = form[0].lower()
                if head == "in-package" and len(form) > 1:
                    cur = name(form[1])
                elif head == "defclass" and cur and len(form) > 3 and isinstance(form[3], list):
                    entry = pkgs.setdefault(cur, {"nicknames": [], "exports": []})
                    entry.setdefault("classes", []).append(name(form[1]))
                    slots = entry.setdefault("slots", [])
                    for slot in form[3]:
                        slots.append(name(slot[0] if isinstance(slot, list) and slot else slot))
            if "defpackage" not in text.lower():
                continue
            todo = list(stack)
            while todo:
                form = todo.pop()
                if not isinstance(form, list) or not form:
                    continue
                head = form[0]
                if isinstance(head, str) and head.lower() == "defpackage" and len(form) > 1:
                    pname = name(form[1])
                    entry = pkgs.setdefault(pname, {"nicknames": [], "exports": []})
                    for opt in form[2:]:
                        if not isinstance(opt, list) or not opt:
                            continue
                        key = name(opt[0])
                        if key == "EXPORT":
                            entry["exports"] += [name(s) for s in opt[1:] if not isinstance(s, list)]
                        elif key == "NICKNAMES":
                            entry["nicknames"] += [name(s) for s in opt[1:] if not isinstance(s, list)]
                else:
                    todo.extend(x for x in form if isinstance(x, list))
    for v in pkgs.values():
        v["exports"] = sorted(set(v["exports"]))
        v["nicknames"] = sorted(set(v["nicknames"]))
        v["slots"] = sorted(set(v.get("slots", [])))
        v["classes"] = sorted(set(v.get("classes", [])))
    with open(os.path.join(HERE, "femlisp_exports.json"), "w") as f:
        json.dump(pkgs, f, indent=0, sort_keys=True)
    print(f"{len(pkgs)} packages")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
