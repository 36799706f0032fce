"""Build tests/golden/reference_declarations.json from the reference's headers.

The reference-side binding in INTEGRATION.md (section 3) is C++ written against the reference's
classes. Their headers include GSL and Boost uBLAS, which this image does not have, so the
binding cannot be compiled here; tests/test_integration_binding.py checks it against the
declarations this script records instead:

* NewtonRaphsonSolver (NewtonRaphsonSolver.h): every member function with its parameter count;
* the members of ShapeBase, Node and ReferenceShapeBase with their access (public / protected /
  private), from their class bodies;
* the NewtonRaphsonSolver methods Simulation::updateStepNR calls (Simulation.cpp).

Run from the repository root with the reference's checkout given:
    REFERENCE_ROOT=<path to the reference> python tests/golden/make_reference_declarations.py
"""
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))


def _strip_comments(text):
    """Comments and preprocessor lines removed (the declarations inside #ifdef blocks are kept)."""
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    return re.sub(r"(?m)^\s*#[^\n]*$", "", text)


def _class_body(text, name):
    m = re.search(r"class\s+" + name + r"\b[^{;]*\{", text)
    depth, i = 1, m.end()
    while depth:
        depth += {"{": 1, "}": -1}.get(text[i], 0)
        i += 1
    return text[m.end():i - 1]


def _members(body):
    """(name, access, n_params or None) of the declarations at the class body's top level."""
    out, access, depth, stmt = [], "private", 0, ""
    for ch in body:
        if ch == "{":
            depth += 1
            continue
        if ch == "}":
            depth -= 1
            if depth == 0:
                stmt = stmt + ";"
            else:
                continue
        if depth:
            continue
        stmt += ch
        if ch in ";:" or stmt.endswith(";"):
            s = stmt.strip()
            if s in ("public:", "protected:", "private:"):
                access = s[:-1]
                stmt = ""
                continue
            if ch == ":" and not s.endswith("::") and "(" not in s and "::" not in s[-2:]:
                continue
            if s.endswith(";"):
                s = s[:-1].strip()
                stmt = ""
                if not s or s.startswith("#") or s.startswith("friend"):
                    continue
                fm = re.search(r"~?\b(\w+)\s*\(([^()]*(?:\([^()]*\)[^()]*)*)\)\s*(const)?\s*(=\s*0)?\s*$", s)
                if fm:
                    params = fm.group(2).strip()
                    n = 0 if params in ("", "void") else len(_split_top(params))
                    out.append((("~" if s.lstrip().startswith("~") or "~" + fm.group(1) in s else "") + fm.group(1),
                                access, n))
                else:
                    for name in re.findall(r"\b(\w+)\s*(?:\[[^\]]*\])*\s*(?:=[^,]*)?(?:,|$)", s.split("=")[0]):
                        out.append((name, access, None))
    return out


def _split_top(params):
    parts, depth, cur = [], 0, ""
    for ch in params:
        if ch in "<(":
            depth += 1
        elif ch in ">)":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    return parts


def main():
    ref = os.environ.get("REFERENCE_ROOT")
    if not ref:
        raise SystemExit("set REFERENCE_ROOT to the reference checkout")
    src = os.path.join(ref, "TissueFolding", "SourceCode")
    out = {}
    for cls, header in (("NewtonRaphsonSolver", "NewtonRaphsonSolver.h"), ("ShapeBase", "ShapeBase.h"),
                        ("Node", "Node.h"), ("ReferenceShapeBase", "ReferenceShapeBase.h")):
        body = _class_body(_strip_comments(open(os.path.join(src, header)).read()), cls)
        out[cls] = [{"name": n, "access": a, "params": p} for n, a, p in _members(body)]
    sim = _strip_comments(open(os.path.join(src, "Simulation.cpp")).read())
    m = re.search(r"void Simulation::updateStepNR\(\)\s*\{", sim)
    depth, i = 1, m.end()
    while depth:
        depth += {"{": 1, "}": -1}.get(sim[i], 0)
        i += 1
    out["updateStepNR_calls"] = sorted(set(re.findall(r"NRSolver->(\w+)\s*\(", sim[m.end():i])))
    path = os.path.join(HERE, "reference_declarations.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(f"wrote {path}: " + ", ".join(f"{k} {len(v)}" for k, v in out.items()))


if __name__ == "__main__":
    main()
