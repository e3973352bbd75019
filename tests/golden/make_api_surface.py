"""Extract the public method surface of the reference's WebGPUEngine class
(src/webgpu-engine.mjs) into webgpu_engine_api.json: name, parameter list as
written, async or not, and the line it starts on.  Methods whose names start
with '_' are private and left out.

Usage: python tests/golden/make_api_surface.py <reference checkout>
The output is committed so the tests never read the reference tree.
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_api_surface.py <path of the reference checkout>")
src = os.path.join(sys.argv[1], "src", "webgpu-engine.mjs")
lines = open(src).read().split("\n")
start = next(i for i, l in enumerate(lines) if re.match(r"^export class WebGPUEngine\b", l))
# the class body ends at the last column-0 "}" (column-0 braces inside WGSL
# template strings end with a backtick or ';')
end = max(i for i in range(start + 1, len(lines)) if lines[i].rstrip() == "}")
pat = re.compile(r"^    (async )?([A-Za-z][A-Za-z0-9_]*)\((.*)\)\s*\{\s*$")
out = []
for i in range(start, end):
    m = pat.match(lines[i])
    if m and m.group(2) not in ("if", "for", "while", "switch", "catch"):
        out.append({"name": m.group(2), "params": m.group(3), "async": bool(m.group(1)), "line": i + 1})
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "webgpu_engine_api.json"), "w") as f:
    json.dump({"source": "src/webgpu-engine.mjs:%d-%d" % (start + 1, end + 1), "methods": out}, f, indent=1)
print("%d public methods" % len(out))
