"""Every reference citation in include/*.h and include/*.hpp lands where it
says, checked against the reference tree the oracle was built from (skipped
where that tree is absent):

  - each `file:lines` names a file of the reference and lines inside it
    (`:lines` continues the file of the previous citation);
  - a citation that follows a qualified name, as in
    `GPU_Implementation6::reset_grid (gpu_implementation6.cpp:18-29)`, has
    that function's name on the first cited line (its definition).
"""
import glob
import os
import re

import pytest

from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = po.reference_tree()
pytestmark = pytest.mark.skipif(REF is None, reason="the reference tree is not on this machine")

CITE = re.compile(r"(?:(?P<file>[\w./]+\.(?:cpp|cu|cuh|h))|(?<![\w.]))"
                  r":(?P<ranges>\d+(?:-\d+)?(?:,\s*\d+(?:-\d+)?)*)")
NAME = re.compile(r"(?P<name>~?\w+(?:::~?\w+)+)\s*$")


def headers():
    return sorted(glob.glob(os.path.join(ROOT, "include", "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.hpp")))


def resolve(name):
    hits = [p for p in glob.glob(os.path.join(REF, "**", os.path.basename(name)), recursive=True)
            if p.replace(os.sep, "/").endswith("/" + name)]
    return hits[0] if len(hits) == 1 else None


def comment_text(path):
    """The header's text with comment leaders removed, lines joined."""
    lines = []
    for ln in open(path):
        ln = re.sub(r"^\s*(/\*+|\*+/?|//+)", " ", ln.rstrip("\n"))
        lines.append(ln)
    return " ".join(lines)


def citations(path):
    """(name or None, file, [(a, b), ...]) per parenthesised citation group."""
    text = comment_text(path)
    out = []
    current = None
    for m in re.finditer(r"\(([^()]*)\)", text):
        group = m.group(1)
        items = list(CITE.finditer(group))
        if not items:
            continue
        nm = NAME.search(text[:m.start()])
        name = nm.group("name") if nm else None
        first = True
        for it in items:
            current = it.group("file") or current
            ranges = []
            for r in it.group("ranges").split(","):
                a, _, b = r.strip().partition("-")
                ranges.append((int(a), int(b or a)))
            out.append((name if first else None, current, ranges))
            first = False
    return out


def bare_citations(path):
    """(file, [(a, b), ...]) for every citation with an explicit file name,
    in parentheses or not."""
    out = []
    for it in CITE.finditer(comment_text(path)):
        if it.group("file"):
            ranges = []
            for r in it.group("ranges").split(","):
                a, _, b = r.strip().partition("-")
                ranges.append((int(a), int(b or a)))
            out.append((it.group("file"), ranges))
    return out


def test_headers_cite_the_reference():
    assert sum(len(citations(h)) for h in headers()) > 30
    assert sum(1 for h in headers() for c in citations(h) if c[0]) > 25


@pytest.mark.parametrize("header", [os.path.basename(h) for h in headers()])
def test_citations_land_on_the_named_lines(header):
    path = os.path.join(ROOT, "include", header)
    bad = []
    for name, fname, ranges in citations(path) + [(None, f, r) for f, r in bare_citations(path)]:
        ref = resolve(fname)
        if ref is None:
            bad.append(f"{fname}: not a file of the reference")
            continue
        lines = open(ref, errors="replace").read().split("\n")
        for a, b in ranges:
            if not (1 <= a <= b <= len(lines)):
                bad.append(f"{fname}:{a}-{b} outside its {len(lines)} lines")
        if name:
            fn = name.split("::")[-1]
            a = ranges[0][0]
            if a <= len(lines) and not re.search(r"(?<![\w~])" + re.escape(fn) + r"\s*\(", lines[a - 1]):
                bad.append(f"{name} ({fname}:{a}): line {a} is `{lines[a - 1].strip()}`")
    assert bad == []
