"""Regenerates tests/golden/scattergather.json from the reference's own
known-answer test (test/scattergather.cpp), read as text.

The reference test places one particle at (3.3, 3.2) on a unit-spacing patch
with origin 0 and tabulates the scatter weights of IntCIC, IntS1 and IntS2
for the edge components (Vcheck: i, j, (ex, ey)) and the cell field (Scheck:
i, j, bz); gathers of a field that is 1 on the support must return 1.
Usage: python tests/golden/make_golden.py <path to the reference checkout>
"""
import argparse
import json
import re
from pathlib import Path

ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
ap.add_argument("reference", type=Path, help="root of the reference checkout (holds test/scattergather.cpp)")
ref = ap.parse_args().reference
src = (ref / "test" / "scattergather.cpp").read_text()

sections = re.split(r"// CHECK (CIC|S1|S2)", src)
out = {"particle": [3.3, 3.2], "origin": [0.0, 0.0], "spacing": [1.0, 1.0],
       "source": "test/scattergather.cpp", "tolerance": 1e-8, "tables": {}}
order = {"CIC": 0, "S1": 1, "S2": 2}
for name, body in zip(sections[1::2], sections[2::2]):
    vc = re.findall(r"Vcheck\((\d+),\s*(\d+),\s*Vector_t\(([-\d.e]+),\s*([-\d.e]+)\)\)", body)
    sc = re.findall(r"Scheck\((\d+),\s*(\d+),\s*([-\d.e]+)\)", body)
    out["tables"][name] = {
        "order": order[name],
        "edge": [[int(i), int(j), float(a), float(b)] for i, j, a, b in vc],
        "cell": [[int(i), int(j), float(v)] for i, j, v in sc],
    }
# test/scattergather.cpp line numbers of the three tables
out["lines"] = {"CIC": "90-100", "S1": "169-187", "S2": "272-311"}
dst = Path(__file__).with_name("scattergather.json")
dst.write_text(json.dumps(out, indent=1) + "\n")
print("wrote", dst, {k: (len(v["edge"]), len(v["cell"])) for k, v in out["tables"].items()})
