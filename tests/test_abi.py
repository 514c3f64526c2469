"""The C-ABI library loads and exports every entry point declared in include/*.h (no GPU
calls are made here)."""
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names |= set(re.findall(r"^EXF_API\s+[\w\s\*]+?\b(exf_\w+)\s*\(", open(h).read(), re.M))
    return names


def test_header_declares_the_api():
    names = declared()
    for n in ("exf_mesh_create", "exf_sys_create", "exf_gen_mat_rhs", "exf_mg_solve", "exf_adjoint_forward",
              "exf_adjoint_backward", "exf_resid", "exf_restrict", "exf_prolong"):
        assert n in names


def test_library_builds_and_exports_every_declared_symbol():
    from exfemus_b200 import build
    so = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s+(exf_\w+)", out))
    missing = declared() - exported
    assert not missing, missing


def test_ctypes_binding_covers_the_header():
    from exfemus_b200 import _lib
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert declared() <= bound
    L = _lib.load()
    for name in declared():
        assert hasattr(L, name)


def test_library_is_built_for_sm100a_only():
    from exfemus_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
