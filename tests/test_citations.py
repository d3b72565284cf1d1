"""Every ``file.py:a-b`` citation of the reference in this repository's
sources points at lines that exist.

The reference's files and their line counts are recorded in
tests/golden/ref_index.json (written by tests/golden/make_ref_index.py from a
checkout of kemi2805/HLLD-AI), so the check needs no reference at run time.
A citation names a file by its path within the reference or by its base
name; bare ``:a-b`` ranges that follow a citation on the same line belong to
the same file.
"""
from __future__ import annotations

import json
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INDEX = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_index.json")))

SOURCES = ["include", "hlld_ai_b200", "oracle", "tests", "bench.py", "__graft_entry__.py",
           "DESIGN.md", "INTEGRATION.md", "README.md"]
EXTS = (".py", ".h", ".cuh", ".cu", ".c", ".cpp", ".md")
# files of this repository that share a base name with a reference file and
# are cited by their repository path
OWN = ("tests/", "hlld_ai_b200/", "oracle/", "include/", "profiles/")

CITE = re.compile(r"(?<![\w/.])((?:[\w.-]+/)*[\w.-]+\.py):(\d+)(?:-(\d+))?")
CONT = re.compile(r"(?<=[\s,(;])?:(\d+)(?:-(\d+))?(?![\d.])")


def _by_base():
    out = {}
    for path, n in INDEX.items():
        out.setdefault(os.path.basename(path), []).append((path, n))
    return out


BASE = _by_base()


def _files():
    for s in SOURCES:
        p = os.path.join(ROOT, s)
        if os.path.isfile(p):
            yield p
            continue
        for dirpath, dirs, files in os.walk(p):
            dirs[:] = [d for d in dirs if d not in ("__pycache__", "golden")]
            for f in files:
                if f.endswith(EXTS):
                    yield os.path.join(dirpath, f)


def _candidates(name):
    if name.startswith(OWN):
        return None
    if name in INDEX:
        return [(name, INDEX[name])]
    for path, n in INDEX.items():
        if path.endswith("/" + name):
            return [(path, n)]
    return BASE.get(os.path.basename(name))


def citations():
    """(source file, line number, cited file, first, last) of every citation."""
    for path in _files():
        rel = os.path.relpath(path, ROOT)
        for ln, line in enumerate(open(path, encoding="utf-8", errors="replace"), 1):
            pos, current = 0, None
            while True:
                m = CITE.search(line, pos)
                nxt = m.start() if m else len(line)
                if current is not None:
                    for c in re.finditer(r"(?:^|[\s,(;])\:(\d+)(?:-(\d+))?", line[pos:nxt]):
                        a = int(c.group(1))
                        yield rel, ln, current, a, int(c.group(2) or a)
                if not m:
                    break
                cands = _candidates(m.group(1))
                current = m.group(1) if cands else None
                if cands:
                    a = int(m.group(2))
                    yield rel, ln, m.group(1), a, int(m.group(3) or a)
                pos = m.end()


def test_reference_citations_point_at_existing_lines():
    bad = []
    n = 0
    for src, ln, name, a, b in citations():
        n += 1
        cands = _candidates(name)
        if not any(1 <= a <= b <= length for _, length in cands):
            bad.append(f"{src}:{ln}: {name}:{a}-{b} (file has {[l for _, l in cands]} lines)")
    assert n > 200, n
    assert not bad, "\n".join(bad)


def test_driver2d_citations_are_inside_the_file():
    lines = [c for c in citations() if c[2].endswith("driver2d.py")]
    assert lines
    assert all(c[4] <= INDEX["src/physics/driver2d.py"] for c in lines)
