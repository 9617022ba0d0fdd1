"""The C-ABI library builds for sm_100a, loads, exports every entry point
declared in include/qmcb200.h, and refuses to run without a CUDA device
(no CPU fallback)."""
import ctypes as C
import os
import re

import pytest
import torch

from qmcbeaver_b200 import build
from qmcbeaver_b200.api import EXPORTS, QMCB200Functions, QMCBError, load_library
from qmcbeaver_b200.system import make_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "qmcb200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(qmcb_[a-z_]+)\s*\(", txt)))


def test_library_builds_and_exports_header():
    path = build.build()
    lib = C.CDLL(path)
    declared = header_functions()
    assert declared, "no functions parsed from the header"
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in qmcb200.h but not exported"
    assert sorted(EXPORTS) == declared


def test_library_is_sm100a():
    path = build.build()
    assert "sm_100a" in " ".join(build.NVCC_FLAGS)
    lib = load_library()
    lib.qmcb_version.restype = C.c_char_p
    assert b"sm_100a" in lib.qmcb_version()
    assert os.path.getsize(path) > 0


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_create_fails_loudly_without_device():
    build.build()
    with pytest.raises(QMCBError, match="no CUDA device"):
        QMCB200Functions(make_system("vmc_water_10e"), 4)


def test_bad_arguments_rejected_before_device_use():
    build.build()
    lib = load_library()
    h = C.c_void_p()
    assert lib.qmcb_create(None, 4, C.byref(h)) == 1  # QMCB_E_ARG
    assert b"null argument" in lib.qmcb_last_error(None)


@pytest.mark.parametrize("cname,pyname", [("qmcb_system_desc", "SystemDesc"), ("qmcb_run_params", "RunParams"),
                                          ("qmcb_step_stats", "StepStats")])
def test_ctypes_mirror_matches_header_layout(tmp_path, cname, pyname):
    """Every field of the ctypes mirrors in qmcbeaver_b200/desc.py sits at the
    offset the C compiler gives it in include/qmcb200.h (and the sizes agree)."""
    import shutil
    import subprocess
    from qmcbeaver_b200 import desc as D
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    st = getattr(D, pyname)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "qmcb200.h"', "int main(void) {",
             f'  printf("%zu\\n", sizeof({cname}));']
    for name, _ in st._fields_:
        lines.append(f'  printf("%zu\\n", offsetof({cname}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call([gcc, "-I", os.path.join(root, "include"), str(src), "-o", str(exe)])
    got = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    assert got[0] == C.sizeof(st), (pyname, got[0], C.sizeof(st))
    for (name, _), off in zip(st._fields_, got[1:]):
        assert getattr(st, name).offset == off, (pyname, name, off)
