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


def test_python_constants_match_the_header_enums():
    """The ctypes binding's misfit kinds, adjoint modes and precisions carry
    the values include/gerjoii_gpu.h gives them, and every obj_FNC name maps
    to a declared misfit kind."""
    import re
    from gerjoii_b200 import _native as N
    hdr = open(os.path.join(ROOT, "include", "gerjoii_gpu.h")).read()
    for name in ("GJ_MISFIT_L2", "GJ_MISFIT_ENV_L2", "GJ_MISFIT_PHASE_L2", "GJ_MISFIT_ENV_L22", "GJ_MISFIT_ENV_LOG",
                 "GJ_ADJ_REFERENCE", "GJ_ADJ_EXACT", "GJ_F32", "GJ_F64"):
        m = re.search(rf"\b{name}\s*=\s*(\d+)", hdr)
        assert m, name
        assert getattr(N, name) == int(m.group(1)), name
    assert set(N.MISFIT_KINDS.values()) == {0, 1, 2, 3, 4}
    assert N.misfit_kind("env_LOG") == N.GJ_MISFIT_ENV_LOG and N.misfit_kind(3) == 3


def test_kernel_kinds_match_the_library_enum():
    """The ctypes binding's kernel-timing kinds carry the numbers the library's
    KernelKind enum gives them (gj_kernel_time's `kind`), the blocked forward
    pass included."""
    from gerjoii_b200 import _native as N
    txt = open(os.path.join(ROOT, "gerjoii_b200", "csrc", "gj_internal.h")).read()
    body = re.search(r"enum KernelKind\s*\{(.*?)\};", txt, flags=re.S).group(1)
    enum = {k: int(v) for k, v in re.findall(r"\b(KK_[A-Z0-9_]+)\s*=\s*(\d+)", body)}
    names = {"fwd_step": "KK_FWD_STEP", "ref_step": "KK_REF_STEP", "adj_step": "KK_ADJ_STEP", "io": "KK_IO",
             "plain": "KK_PLAIN", "dc_factor": "KK_DC_FACTOR", "image": "KK_IMAGE", "dc_precond": "KK_DC_PRECOND",
             "tb_pass": "KK_TB_PASS"}
    assert set(N.Context.KERNEL_KINDS) == set(names)
    for py, c in names.items():
        assert N.Context.KERNEL_KINDS[py] == enum[c], py
    assert enum["KK_NKINDS"] == len(names)
