"""Writes reference_index.json: the line count of every text file of a
SCEMonteCarlo.jl checkout and the definitions (functions, structs, constants, kernels)
of its Julia files with their line numbers. tests/test_citations.py checks every
`path:line` citation in this repository against it, so the tests need no checkout.

  python tests/golden/extract_reference_index.py <SCEMonteCarlo.jl checkout>
"""
import json
import pathlib
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python extract_reference_index.py <SCEMonteCarlo.jl checkout>")
REF = pathlib.Path(sys.argv[1])
DEF = re.compile(r"^\s*(?:@\w+\s+)*(?:function|struct|mutable struct|const|macro|abstract type)\s+"
                 r"([A-Za-z_][\w!.]*)|^\s*(?:@inline\s+)?([A-Za-z_][\w!.]*)\([^)]*\)(?:::[\w{}]+)?\s*=")
files = {}
for p in sorted(REF.rglob("*")):
    if not p.is_file() or ".git" in p.parts:
        continue
    try:
        text = p.read_text()
    except (UnicodeDecodeError, OSError):
        continue
    lines = text.splitlines()
    entry = {"lines": len(lines)}
    if p.suffix == ".jl":
        defs = []
        for i, line in enumerate(lines, 1):
            m = DEF.match(line)
            if m:
                name = m.group(1) or m.group(2)
                defs.append([i, name.split(".")[-1]])
        entry["defs"] = defs
    files[str(p.relative_to(REF))] = entry
dst = pathlib.Path(__file__).with_name("reference_index.json")
dst.write_text(json.dumps({"source": "SCEMonteCarlo.jl v0.1.0 checkout", "files": files}, indent=0) + "\n")
print(dst, len(files), "files")
