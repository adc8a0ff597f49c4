"""Writes tests/golden/dc_corner_manifold.json: the reference's corner-
manifold table of the dual-contouring collapse test (DCTree<3>::
cornersAreManifold, libfive/src/render/brep/dc/dc_tree3.cpp:111-154), read
as text from the 256-entry literal in the reference source.

    python tests/golden/make_dc_manifold_fixture.py /root/reference
"""
import json
import os
import re
import sys

ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
src = os.path.join(ref, "libfive", "src", "render", "brep", "dc", "dc_tree3.cpp")
text = open(src).read()
m = re.search(r"corner_table\[\]\s*=\s*\{([^}]*)\}", text)
bits = [int(b) for b in re.findall(r"[01]", m.group(1))]
assert len(bits) == 256
line = text[:m.start()].count("\n") + 1
out = {"_source": "libfive/src/render/brep/dc/dc_tree3.cpp:%d (cornersAreManifold)" % line,
       "manifold": bits}
here = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(here, "dc_corner_manifold.json"), "w") as f:
    json.dump(out, f)
    f.write("\n")
print("wrote", len(bits), "entries from", out["_source"])
