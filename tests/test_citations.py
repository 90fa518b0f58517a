"""Every `path:line` citation of the reference in this repository points at lines
that exist, and each entry of include/scemc.h's interface table names a function
defined in the lines it cites.

The reference's file lengths and definitions come from tests/golden/
reference_index.json (written by tests/golden/extract_reference_index.py from a
checkout), so the test needs no checkout.
"""
import json
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
INDEX = json.loads((ROOT / "tests" / "golden" / "reference_index.json").read_text())["files"]

# the files of this repository that cite the reference
SOURCES = sorted({*ROOT.glob("include/*.h"), *ROOT.glob("scemontecarlo.jl_b200/*.py"),
                  *ROOT.glob("scemontecarlo.jl_b200/csrc/*"), *ROOT.glob("oracle/*.cpp"), *ROOT.glob("oracle/*.py"),
                  *ROOT.glob("tests/*.py"), *ROOT.glob("tests/golden/*.py"), ROOT / "bench.py",
                  ROOT / "__graft_entry__.py", ROOT / "DESIGN.md", ROOT / "INTEGRATION.md", ROOT / "README.md"})
CITE = re.compile(r"(?<![\w/.-])((?:[\w.-]+/)*[\w.-]+\.(?:jl|md|toml|yml))((?::\d+(?:-\d+)?)(?:,\d+(?:-\d+)?)*)")


def resolve(cited: str):
    """The index key of a cited reference path (full relative path or a unique suffix)."""
    if cited in INDEX:
        return cited
    hits = [k for k in INDEX if k.endswith("/" + cited)]
    return hits[0] if len(hits) == 1 else None


def citations():
    out = []
    for src in SOURCES:
        if not src.is_file():
            continue
        for no, line in enumerate(src.read_text(errors="replace").splitlines(), 1):
            for m in CITE.finditer(line):
                out.append((src.relative_to(ROOT).as_posix(), no, m.group(1), m.group(2)))
    return out


def ranges(spec: str):
    for part in spec.lstrip(":").split(","):
        a, _, b = part.partition("-")
        yield int(a), int(b or a)


def test_index_covers_the_sweep_path():
    for f in ("src/gpu/gpu_sweep.jl", "src/gpu/gpu_state.jl", "src/gpu/gpu_hamiltonian.jl", "src/updates.jl",
              "src/energy.jl", "src/hamiltonian.jl", "test/unit/test_gpu.jl"):
        assert INDEX[f]["lines"] > 50


def test_every_reference_citation_exists():
    bad, n = [], 0
    for src, no, path, spec in citations():
        key = resolve(path)
        if key is None:
            # a .jl file is always the reference's; other files may be this repository's own
            if path.endswith(".jl"):
                bad.append(f"{src}:{no}: {path} is not a reference file (or is ambiguous)")
            continue
        n += 1
        for a, b in ranges(spec):
            if not (1 <= a <= b <= INDEX[key]["lines"]):
                bad.append(f"{src}:{no}: {path}:{a}-{b} outside {key} ({INDEX[key]['lines']} lines)")
    assert n > 100
    assert not bad, "\n".join(bad)


HEADER_ROW = re.compile(r"^ \*\s+(scemc_\w+\*?)\s+([A-Za-z_][\w!]*).*?\s((?:src|test)/[\w/]+\.jl):(\d+)-(\d+)\s*$")


def test_header_interface_table_names_the_cited_functions():
    text = (ROOT / "include" / "scemc.h").read_text().splitlines()
    rows = [m for m in (HEADER_ROW.match(l) for l in text) if m]
    assert len(rows) >= 11
    for m in rows:
        entry, name, path, a, b = m.group(1), m.group(2), m.group(3), int(m.group(4)), int(m.group(5))
        ident = name
        defs = INDEX[path]["defs"]
        inside = {d for ln, d in defs if a <= ln <= b}
        assert ident in inside, f"{entry}: {ident} is not defined in {path}:{a}-{b} (defined there: {sorted(inside)})"


def test_overrelaxation_row_cites_the_cpu_sweep():
    text = (ROOT / "include" / "scemc.h").read_text()
    assert re.search(r"scemc_overrelaxation_sweep.*\n.*src/updates\.jl:231-248", text)


if __name__ == "__main__":
    pytest.main([__file__, "-q"])
