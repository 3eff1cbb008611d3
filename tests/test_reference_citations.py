"""Every reference citation in the product, the oracle, the tests and the
integration documents points at lines that exist in the reference, and a
citation written next to the name of a reference function or type covers that
definition's first line.

This reads the reference project's sources (the directory in the environment
variable FFCM_REFERENCE_ROOT, by default the read-only checkout the build
container holds) and is skipped where that checkout is absent.
"""
from __future__ import annotations

import os
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
REF = Path(os.environ.get("FFCM_REFERENCE_ROOT", "/root/reference"))

pytestmark = pytest.mark.skipif(not (REF / "src" / "mobility.jl").exists(),
                                reason="the reference sources are not present on this machine")

# file:line or file:a-b, optionally followed by ", c-d" ranges of the same file
CITE = re.compile(r"((?:src|ext|test|docs|benchmark)/[\w/.\-]+?\.(?:jl|md|toml))"
                  r"((?::\d+(?:-\d+)?)(?:,\s*:?\d+(?:-\d+)?)*)?")
# definitions: `function name`, `struct Name`, `name(...) = ` one-liners
DEF = re.compile(r"^(?:@inline\s+)?(?:function|struct|mutable struct)\s+([\w.!:]+?)[({\s]|^([\w!]+)\(.*\)\s*=")


def _cited_files():
    out = subprocess.run(["git", "ls-files"], cwd=ROOT, capture_output=True, text=True, check=True).stdout.split()
    skip = ("VERDICT", "ADVICE", "SURVEY", "BASELINE", "GPUTEST", "BENCH", "MULTICHIP", "SCALE", "PROGRESS")
    keep = []
    for f in out:
        # this file's own examples are patterns, not citations
        if f.startswith(skip) or f.endswith((".npz", ".json")) or f.endswith("test_reference_citations.py"):
            continue
        keep.append(ROOT / f)
    return keep


def _citations():
    found = []
    for f in _cited_files():
        if not f.is_file():
            continue
        text = f.read_text(errors="replace")
        for m in CITE.finditer(text):
            ranges = []
            for part in re.findall(r"\d+(?:-\d+)?", m.group(2) or ""):
                a, _, b = part.partition("-")
                ranges.append((int(a), int(b or a)))
            # the identifier written closest before the citation, same line
            line_start = text.rfind("\n", 0, m.start()) + 1
            before = text[line_start:m.start()]
            found.append((f.relative_to(ROOT), m.group(1), ranges, before))
    return found


def _definitions(path):
    defs = {}
    for i, line in enumerate(path.read_text(errors="replace").splitlines(), 1):
        d = DEF.match(line)
        if d:
            name = (d.group(1) or d.group(2)).split("{")[0]
            defs.setdefault(name, []).append(i)
    return defs


def test_citations_exist_and_stay_in_range():
    cites = _citations()
    assert len(cites) > 150        # the product cites the reference throughout
    bad = []
    for src, path, ranges, _ in cites:
        ref = REF / path
        if not ref.exists():
            # the Julia extension a maintainer would add is named, not cited
            if "B200Ext" in path:
                continue
            bad.append(f"{src}: {path} does not exist")
            continue
        n = len(ref.read_text(errors="replace").splitlines())
        for a, b in ranges:
            if not (1 <= a <= b <= n):
                bad.append(f"{src}: {path}:{a}-{b} outside 1-{n}")
    assert not bad, "\n".join(bad)


def test_citations_next_to_a_definition_cover_it():
    """`name!` (src/x.jl:a-b): the definition of name! starts inside a-b."""
    checked, bad = 0, []
    defs_cache = {}
    for src, path, ranges, before in _citations():
        ref = REF / path
        if not ranges or not ref.exists() or not path.endswith(".jl"):
            continue
        defs = defs_cache.setdefault(path, _definitions(ref))
        names = re.findall(r"[`\s(]([A-Za-z_][\w!]*!?)(?:\{T\})?(?:\([^()]*\))?`?", " " + before)
        names = [x for x in names if x in defs]
        if not names:
            continue
        name = names[-1]
        checked += 1
        lines = defs[name]
        if not any(a <= ln <= b for ln in lines for a, b in ranges):
            bad.append(f"{src}: `{name}` cited as {path}:{ranges} but defined at line(s) {lines}")
    assert checked >= 25
    assert not bad, "\n".join(bad)
