"""Every `file:line` citation of the reference in this repository's sources and notes resolves.

A citation names a reference file by its path within the reference project (or a unique tail of
it) followed by line numbers or ranges, e.g. ``Core/PartSpecies.cc:105-109, 147-159``; a bare
``:N`` or ``:N-M`` later on the same line continues the last file named there.  The test
finds each one, resolves the file inside the reference tree given by the environment variable
H1D_REFERENCE, and checks that every cited line exists in that file and that ranges are ordered.
Files of this repository (the CUDA sources, the oracle, the tests) are recognised by name and
skipped.  Without H1D_REFERENCE the test is skipped: the reference tree is not part of this
repository.
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("H1D_REFERENCE")

CITE = re.compile(r"(?<![\w/.-])((?:[A-Za-z0-9_-]+/)*[A-Za-z0-9_-]+\.(?:cc|hh|h|txt|md)):"
                  r"(\d+(?:-\d+)?(?:,\s*\d+(?:-\d+)?)*)")
BARE = re.compile(r"(?<=[\s(`]):(\d+(?:-\d+)?(?:,\s*\d+(?:-\d+)?)*)")
# sources of this repository that may be cited with line numbers too
OWN = {"h1d_gpu.h", "h1d_oracle.c", "ref_driver.cc", "HDF5Kit.h", "DESIGN.md", "INTEGRATION.md", "README.md",
       "Inputs.h.in", "Domain_GPU.h", "Domain_GPU.cc"}
SCANNED_DIRS = ("hybrid_code-hfemic_wave_b200", "include", "oracle", "tests", "adapter")
SCANNED_TOP = ("bench.py", "__graft_entry__.py", "DESIGN.md", "INTEGRATION.md", "README.md")
SUFFIXES = (".py", ".cu", ".cuh", ".h", ".hh", ".cc", ".c", ".md", "Makefile")


def _reference_files():
    files = {}
    for d, _, names in os.walk(REF):
        if "/.git" in d:
            continue
        for n in names:
            rel = os.path.relpath(os.path.join(d, n), REF)
            files[rel] = os.path.join(d, n)
    return files


def _resolve(cited, files):
    """The reference file a citation names: the paths ending in the cited path; when several do,
    the one in the hybrid code or the non-relativistic LibPIC tree (runs and the relativistic VDFs
    are cited with their directory)."""
    tail = "/" + cited
    cands = [r for r in files if ("/" + r).endswith(tail)]
    if len(cands) > 1:
        cands = [r for r in cands if "RelativisticVDF/" not in r and not r.startswith("00-runs/")] or cands
    return cands[0] if len(cands) == 1 else (None if not cands else cands)


def _scanned():
    out = [os.path.join(ROOT, f) for f in SCANNED_TOP]
    for top in SCANNED_DIRS:
        base = os.path.join(ROOT, top)
        for d, dirs, names in os.walk(base):
            dirs[:] = [x for x in dirs if x not in ("_ref", "_build", "__pycache__", "golden")]
            out += [os.path.join(d, n) for n in names if n.endswith(SUFFIXES)]
    return [p for p in out if os.path.isfile(p) and not p.endswith("test_citations.py")]


def _lines(path, cache={}):
    if path not in cache:
        with open(path, "rb") as f:
            cache[path] = f.read().count(b"\n") + 1
    return cache[path]


def citations():
    files = _reference_files()
    for path in _scanned():
        with open(path, encoding="utf-8", errors="replace") as f:
            text = f.read()
        for m in CITE.finditer(text):
            name = m.group(1)
            if os.path.basename(name) in OWN:
                continue
            line = text.count("\n", 0, m.start()) + 1
            yield os.path.relpath(path, ROOT), line, name, m.group(2), files
            # bare continuations on the same line: "... Foo.cc:12-30 ... :41" cite Foo.cc too
            eol = text.find("\n", m.end())
            rest = text[m.end():eol if eol >= 0 else len(text)]
            stop = CITE.search(rest)
            for b in BARE.finditer(rest[:stop.start()] if stop else rest):
                yield os.path.relpath(path, ROOT), line, name, b.group(1), files


@pytest.mark.skipif(not REF or not os.path.isdir(REF or ""), reason="H1D_REFERENCE (the reference tree) not set")
def test_every_citation_resolves():
    bad, n = [], 0
    for where, line, name, ranges, files in citations():
        n += 1
        rel = _resolve(name, files)
        if rel is None:
            bad.append(f"{where}:{line}: {name} is not a file of the reference")
            continue
        if isinstance(rel, list):
            bad.append(f"{where}:{line}: {name} is ambiguous: {rel}")
            continue
        count = _lines(files[rel])
        for part in ranges.split(","):
            a, _, b = part.strip().partition("-")
            lo, hi = int(a), int(b or a)
            if not 1 <= lo <= hi <= count:
                bad.append(f"{where}:{line}: {name}:{part.strip()} outside 1..{count} of {rel}")
    print(f"{n} citations checked")
    assert n > 100
    assert not bad, "\n".join(bad)
