"""Static checks of the reference-side binding in INTEGRATION.md section 3.

The binding replaces the bodies of the NewtonRaphsonSolver methods Simulation::updateStepNR calls
with forwards to the C ABI. It cannot be compiled in this image (the reference's headers include
GSL and Boost uBLAS, absent here), so it is checked against the reference's declarations recorded
in tests/golden/reference_declarations.json (made by tests/golden/make_reference_declarations.py)
and against include/tf_b200.h:

* every NewtonRaphsonSolver member function it defines is declared in NewtonRaphsonSolver.h with
  as many parameters (or added by the patch's header lines);
* every method updateStepNR calls is either redefined or named as kept from the reference;
* every member it reads on an element, a node or a reference shape is public there (or is an
  accessor the patch adds), and every NewtonRaphsonSolver member it uses is declared;
* every tf_* call names a function of include/tf_b200.h with as many arguments.
"""
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _decls():
    return json.load(open(os.path.join(HERE, "golden", "reference_declarations.json")))


def _section3():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    sec = text[text.index("## 3."):text.index("## 4.")]
    blocks = [re.sub(r"//[^\n]*", "", b) for b in re.findall(r"```cpp\n(.*?)```", sec, flags=re.S)]
    return sec, blocks


def _split_args(s):
    s = s.replace("->", ".")  # member access, not a template bracket
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch in "(<[{":
            depth += 1
        elif ch in ")>]}":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        parts.append(cur)
    return parts


def _calls(code, name_re):
    """(name, argument string) of every call matching name_re, with balanced parentheses."""
    out = []
    for m in re.finditer(name_re + r"\s*\(", code):
        i, depth = m.end(), 1
        while depth:
            depth += {"(": 1, ")": -1}.get(code[i], 0)
            i += 1
        out.append((m.group(1), code[m.end():i - 1]))
    return out


def _header_functions():
    text = open(os.path.join(ROOT, "include", "tf_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(tf_\w+)\s*\(([^;{]*)\)\s*;", text):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else len(_split_args(params))
    return out


def test_defined_methods_are_declared_by_the_reference():
    d = _decls()
    sec, blocks = _section3()
    code = "\n".join(blocks)
    declared = {}
    for m in d["NewtonRaphsonSolver"]:
        if m["params"] is not None:
            declared.setdefault(m["name"], set()).add(m["params"])
    added = set(re.findall(r"void\s+(\w+)\s*\(", blocks[1]))  # the header patch's new members
    assert added == {"gpuUploadStep"}
    defined = _calls(code, r"NewtonRaphsonSolver::(~?\w+)")
    assert defined, "no method definitions found"
    for name, params in defined:
        n = len(_split_args(params))
        if name in added:
            continue
        assert name in declared, name
        assert n in declared[name], (name, n, declared[name])


def test_every_method_updateStepNR_calls_is_covered():
    d = _decls()
    sec, blocks = _section3()
    defined = {n for n, _ in _calls("\n".join(blocks), r"NewtonRaphsonSolver::(~?\w+)")}
    kept_text = sec[sec.index("every other method"):sec.index("```cpp", sec.index("every other method"))]
    kept = set(re.findall(r"`(\w+)`", kept_text))
    numerical = {"useNumericalJacobianInIteration", "calculateDifferenceBetweenNumericalAndAnalyticalJacobian"}
    for name in d["updateStepNR_calls"]:
        assert name in defined or name in kept or name in numerical, name


def test_members_read_are_accessible():
    d = _decls()
    sec, blocks = _section3()
    code = "\n".join(blocks)
    public = {cls: {m["name"] for m in d[cls] if m["access"] == "public"} for cls in ("ShapeBase", "Node", "ReferenceShapeBase")}
    accessors = set(re.findall(r"double\s+(\w+)\(\)\s*const", blocks[0]))
    assert accessors == {"getLambda", "getMu"}
    for name in re.findall(r"Elements\[\w+\]->(\w+)", code):
        assert name in public["ShapeBase"] or name in accessors, name
    for name in re.findall(r"Nodes\[\w+\]->(\w+)", code):
        assert name in public["Node"], name
    for name in re.findall(r"ReferenceShape->(\w+)", code):
        assert name in public["ReferenceShapeBase"], name
    members = {m["name"] for m in d["NewtonRaphsonSolver"]}
    body = blocks[2]
    for name in ("threshold", "nDim", "nNodes", "un", "uk", "deltaU", "gExt", "gSum", "K", "Knumerical",
                 "slaveMasterList", "displacementPerDt", "boundNodesWithSlaveMasterDefinition"):
        if re.search(r"\b" + name + r"\b", body):
            assert name in members, name


def test_abi_calls_match_the_header():
    sec, blocks = _section3()
    funcs = _header_functions()
    calls = _calls("\n".join(blocks), r"\b(tf_\w+)")
    assert {n for n, _ in calls} >= {"tf_create", "tf_newton_iteration", "tf_set_external_force", "tf_set_boundary"}
    for name, args in calls:
        assert name in funcs, name
        assert len(_split_args(args)) == funcs[name], (name, args)
