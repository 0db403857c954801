"""C-ABI library checks that need no GPU: it loads, exports every symbol the
headers declare, and its signatures are registered."""
import glob
import os
import re

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(gj_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_library_builds_and_exports_every_declared_symbol():
    from gerjoii_b200 import build, _native
    build.build()
    lib = _native.load()
    declared = _declared()
    assert declared, "no declarations found in include/*.h"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_native.SIGNATURES) >= declared


def test_version_and_context_without_gpu():
    from gerjoii_b200 import _native
    lib = _native.load()
    assert b"sm_100a" in lib.gj_version()
    # gj_last_error on a null context returns a message, not a crash
    assert lib.gj_last_error(None) == b"null context"


def test_library_has_no_torch_dependency():
    from gerjoii_b200 import build
    with open(build.LIB, "rb") as f:
        blob = f.read()
    assert b"libtorch" not in blob and b"libc10" not in blob
