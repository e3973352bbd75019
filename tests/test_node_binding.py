"""The Node.js drop-in (node/cuda-engine.mjs over node/efs_napi.cc) against
the reference's WebGPUEngine surface and against include/efs.h, on the CPU.

No JavaScript runtime or Node-API headers are installed here, so the binding
is checked statically:
* every public method of WebGPUEngine (tests/golden/webgpu_engine_api.json,
  extracted from src/webgpu-engine.mjs by tests/golden/make_api_surface.py)
  exists in the JS class with the same parameter list (extra trailing
  parameters only with defaults), async where the reference's is;
* every addon.* call of the JS class is a function the addon exports;
* every efs_* function the addon calls is declared in include/efs.h;
* configurePBC forwards each entry's axis and phase (the reference's
  {axes: [{axis, phase}]}, src/webgpu-engine.mjs:1966-1976).
"""
import json
import os
import re

from conftest import ROOT

JS = os.path.join(ROOT, "node", "cuda-engine.mjs")
CC = os.path.join(ROOT, "node", "efs_napi.cc")
HDR = os.path.join(ROOT, "include", "efs.h")


def js_methods():
    src = open(JS).read()
    body = src[src.index("export class WebGPUEngine"):]
    out = {}
    for m in re.finditer(r"^    (async )?(get |set )?([A-Za-z][A-Za-z0-9_]*)\((.*)\)\s*\{", body, re.M):
        if m.group(2):
            continue
        out[m.group(3)] = (m.group(4), bool(m.group(1)))
    return src, out


def split_params(p):
    out, depth, cur = [], 0, ""
    for ch in p:
        if ch in "{[(":
            depth += 1
        elif ch in "}])":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return [re.sub(r"\s+", " ", x) for x in out]


def test_every_public_method_with_the_same_arguments():
    ref = json.load(open(os.path.join(ROOT, "tests", "golden", "webgpu_engine_api.json")))["methods"]
    _, ours = js_methods()
    assert len(ref) >= 40
    for m in ref:
        assert m["name"] in ours, "missing method %s (reference line %d)" % (m["name"], m["line"])
        params, is_async = ours[m["name"]]
        rp, op = split_params(m["params"]), split_params(params)
        assert op[:len(rp)] == rp, (m["name"], rp, op)
        assert all("=" in x for x in op[len(rp):]), (m["name"], op)
        if m["name"] != "constructor":
            assert is_async == m["async"], m["name"]


def test_addon_calls_resolve_to_exports_and_header():
    src, _ = js_methods()
    calls = set(re.findall(r"\baddon\.([A-Za-z]+)\(", src))
    cc = open(CC).read()
    exported = set(re.findall(r'\{"([A-Za-z]+)", nullptr, [A-Za-z]+,', cc))
    assert calls and calls <= exported, calls - exported
    used = set(re.findall(r"\b(efs_[a-z_]+)\(", cc))
    hdr = open(HDR).read()
    declared = set(re.findall(r"\b(efs_[a-z_]+)\(", hdr))
    assert used <= declared, used - declared


def test_pbc_entries_carry_axis_and_phase():
    src, _ = js_methods()
    body = src[src.index("    configurePBC(config) {"):]
    body = body[:body.index("\n    }\n")]
    assert "a.axis" in body and "a.phase" in body
