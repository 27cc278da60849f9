"""Every `file.jl:N` citation in the product, the oracle, the tests and the docs
must point inside the cited file of the reference (IBPM.jl).  The reference
tree is taken from $IBPM_REFERENCE_ROOT, else from a `reference` directory
beside the repository's parent; without it the test is skipped (the GPU box
has no copy of the reference)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SCAN_DIRS = ["include", "oracle", "ibpm.jl_b200", "tests"]
SCAN_FILES = ["DESIGN.md", "INTEGRATION.md", "README.md", "bench.py", "__graft_entry__.py"]
EXTS = (".py", ".cu", ".cuh", ".h", ".jl", ".md")
CITE = re.compile(r"([A-Za-z0-9_./-]*\.jl):(\d+)(?:-(\d+))?((?:,\s?\d+(?:-\d+)?)*)")


def reference_root():
    cand = os.environ.get("IBPM_REFERENCE_ROOT") or os.path.join(os.path.dirname(ROOT), "reference")
    return cand if os.path.isdir(os.path.join(cand, "src")) else None


def scanned_files():
    for d in SCAN_DIRS:
        for dp, _, fns in os.walk(os.path.join(ROOT, d)):
            for fn in fns:
                if fn.endswith(EXTS):
                    yield os.path.join(dp, fn)
    for fn in SCAN_FILES:
        p = os.path.join(ROOT, fn)
        if os.path.exists(p):
            yield p


def jl_index(ref):
    """basename -> [(relative path, line count)] over the reference's .jl files."""
    idx = {}
    for dp, _, fns in os.walk(ref):
        for fn in fns:
            if fn.endswith(".jl"):
                p = os.path.join(dp, fn)
                with open(p, encoding="utf-8", errors="replace") as f:
                    n = sum(1 for _ in f)
                idx.setdefault(fn, []).append((os.path.relpath(p, ref), n))
    return idx


def citations(path):
    with open(path, encoding="utf-8", errors="replace") as f:
        for lineno, line in enumerate(f, 1):
            for m in CITE.finditer(line):
                nums = [int(m.group(2))] + ([int(m.group(3))] if m.group(3) else [])
                for extra in re.findall(r"\d+(?:-\d+)?", m.group(4) or ""):
                    nums += [int(x) for x in extra.split("-")]
                yield lineno, m.group(1), nums


def test_every_reference_citation_is_in_range():
    ref = reference_root()
    if ref is None:
        pytest.skip("reference tree not available")
    idx = jl_index(ref)
    bad, n = [], 0
    for p in scanned_files():
        if os.path.abspath(p) == os.path.abspath(__file__):
            continue
        for lineno, name, nums in citations(p):
            base = os.path.basename(name)
            if base not in idx:
                continue   # a file of this repository (the Julia shim), not of the reference
            cands = [(rp, cnt) for rp, cnt in idx[base] if rp.endswith(name) or "/" not in name]
            n += 1
            if not cands or not any(max(nums) <= cnt for _, cnt in cands):
                bad.append("%s:%d cites %s:%s (file has %s lines)"
                           % (os.path.relpath(p, ROOT), lineno, name, nums, [c for _, c in cands]))
    assert n > 50, "too few citations found (%d): is the pattern right?" % n
    assert not bad, "\n".join(bad)
