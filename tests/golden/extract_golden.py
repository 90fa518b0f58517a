"""Extracts the known-answer vectors that SCEMonteCarlo.jl's own test suite holds
for the sweep path into philox_kat.json (run once, with the path of a checkout of
the reference as its argument; the tests read only the JSON).

Source: test/unit/test_gpu.jl:49-59 — the Random123 philox4x32-10 known answers
the reference gates its keyed RNG on — and the open-interval edge words of
test_gpu.jl:70-71.
"""
import json
import pathlib
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python extract_golden.py <SCEMonteCarlo.jl checkout>")
REF = pathlib.Path(sys.argv[1])
src = (REF / "test" / "unit" / "test_gpu.jl").read_text()
hexes = r"\((0x[0-9a-f]+), (0x[0-9a-f]+), (0x[0-9a-f]+), (0x[0-9a-f]+)\)"
pat = re.compile(r"MC\._philox4x32\(" + hexes + r",\s*\((0x[0-9a-f]+), (0x[0-9a-f]+)\)\)\s*==\s*" + hexes)
kats = []
for m in pat.finditer(src):
    g = [int(x, 16) for x in m.groups()]
    kats.append({"ctr": g[0:4], "key": g[4:6], "out": g[6:10]})
assert len(kats) == 3, kats
edges = re.findall(r"MC\._philox_uniform\((0x[0-9a-f]+), (0x[0-9a-f]+)\)", src)
out = {
    "source": "SCEMonteCarlo.jl test/unit/test_gpu.jl:49-71",
    "philox4x32_10": kats,
    "uniform_edge_words": [[int(a, 16), int(b, 16)] for a, b in edges],
}
dst = pathlib.Path(__file__).with_name("philox_kat.json")
dst.write_text(json.dumps(out, indent=1) + "\n")
print(dst, len(kats), "vectors")
