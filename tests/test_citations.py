"""Every natinterp3d citation (file:line or file:line-line) in the C-ABI
header, the integration notes and the product sources points at lines that
exist in natinterp3d's source files.  A bare ":N" right after a citation on
the same line refers to the same file.  Needs natinterp3d's sources (the
NATINTERP3D_ROOT environment variable, else the checkout the build recipes
read); skipped where they are absent."""
import glob
import os
import re

import pytest

from natinterp3d_b200 import _build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_root():
    env = os.environ.get('NATINTERP3D_ROOT')
    if env:
        return env
    src = _build.ref_source_dir()
    # <root>/src/natinterp3d
    return os.path.dirname(os.path.dirname(src)) if src else None


def _reference_files(root):
    """basename -> line count, for names that occur once in natinterp3d's tree"""
    seen = {}
    for dirpath, _, files in os.walk(root):
        for f in files:
            if f.endswith(('.c', '.h', '.pyx', '.py', '.rst', '.toml')):
                seen.setdefault(f, []).append(os.path.join(dirpath, f))
    out = {}
    for name, paths in seen.items():
        if len(paths) == 1:
            with open(paths[0], 'rb') as fh:
                out[name] = fh.read().count(b'\n') + 1
    return out


CITE = re.compile(r'([A-Za-z_][\w-]*\.(?:c|h|pyx|py|rst|toml)):(\d+)(?:-(\d+))?((?:,\s*\d+(?:-\d+)?)*)'
                  r'|(?<=[\s(,`]):(\d+)(?:-(\d+))?')


def _sources():
    pats = ['include/*.h', 'INTEGRATION.md', 'natinterp3d_b200/*.py', 'natinterp3d_b200/csrc/*',
            'oracle/*.c', 'oracle/*.py', 'bench.py', '__graft_entry__.py']
    for pat in pats:
        for p in sorted(glob.glob(os.path.join(ROOT, pat))):
            if os.path.isfile(p):
                yield p


def test_reference_citations_resolve():
    root = _reference_root()
    if not root or not os.path.isdir(root):
        pytest.skip("natinterp3d's sources are not present")
    nlines = _reference_files(root)
    assert 'natural_insertionfree.c' in nlines
    bad, checked = [], 0
    for path in _sources():
        with open(path, encoding='utf-8', errors='replace') as fh:
            for ln, line in enumerate(fh, 1):
                last = None
                for m in CITE.finditer(line):
                    if m.group(1):
                        last = m.group(1)
                        spans = [(m.group(2), m.group(3))]
                        spans += re.findall(r'(\d+)(?:-(\d+))?', m.group(4) or '')
                    else:
                        if last is None:
                            continue
                        spans = [(m.group(5), m.group(6))]
                    if last not in nlines:
                        continue  # not a natinterp3d file (or an ambiguous name)
                    for a, b in spans:
                        a, b = int(a), int(b) if b else int(a)
                        checked += 1
                        if not (1 <= a <= b <= nlines[last]):
                            bad.append('%s:%d cites %s:%d-%d (file has %d lines)'
                                       % (os.path.relpath(path, ROOT), ln, last, a, b, nlines[last]))
    assert checked > 50
    assert not bad, '\n'.join(bad)
