"""CPU checks of the C-ABI library (no GPU): it loads, exports every symbol that
include/*.h declares, and rejects invalid arguments on the host side."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def declared_symbols():
    names = []
    for fn in sorted(os.listdir(INC)):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(INC, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"MM_API\s+[\w\s\*]+?\b(\w+)\s*\(", src):
            names.append(m.group(1))
    return names


def test_header_declares_symbols():
    names = declared_symbols()
    assert "mm_plan_create" in names and "torqueAsync" in names and "zhangli_async" in names
    assert len(names) == len(set(names))


def test_library_exports_every_declared_symbol():
    from mumax2 import _native as nat
    lib = nat.lib()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_strings():
    from mumax2 import _native as nat
    lib = nat.lib()
    assert b"sm_100a" in lib.mm_version()
    assert isinstance(lib.mm_last_error(), bytes)


def test_invalid_arguments_are_rejected_without_a_gpu():
    from mumax2 import _native as nat
    lib = nat.lib()
    h = C.c_void_p()
    assert lib.mm_plan_create(None, C.byref(h)) == nat.MM_ERR_ARG
    p = nat.make_problem(dict(n=(1, 4, 4), cell=(1e-9, 1e-9, 1e-9), msat=0.0))
    assert lib.mm_plan_create(C.byref(p), C.byref(h)) == nat.MM_ERR_ARG
    assert b"Msat" in lib.mm_last_error()
    p = nat.make_problem(dict(n=(1, 0, 4), cell=(1e-9, 1e-9, 1e-9)))
    assert lib.mm_plan_create(C.byref(p), C.byref(h)) == nat.MM_ERR_ARG
    assert lib.mm_solver_init(None, 0, 1e-15, 1e-15, 1e-10, 1e-3) == nat.MM_ERR_ARG
    assert lib.mm_run(None, 1e-9, None) == nat.MM_ERR_ARG


def test_problem_struct_layout_matches_oracle():
    """The product's mm_problem and the oracle's or_desc share their field layout, so
    a test can describe one problem to both."""
    import oracle as O
    from mumax2 import _native as nat
    a = [(n, t) for n, t in nat.MMProblem._fields_]
    b = [(n, t) for n, t in O.OrDesc._fields_]
    assert [x[0] for x in a] == [x[0] for x in b]
    assert C.sizeof(nat.MMProblem) == C.sizeof(O.OrDesc)


@pytest.mark.parametrize("hdr", ["mm_b200.h", "libmumax2_compat.h"])
def test_headers_compile_as_c(hdr, tmp_path):
    import subprocess
    src = tmp_path / "t.c"
    src.write_text(f'#include "{hdr}"\nint main(void){{return 0;}}\n')
    r = subprocess.run(["gcc", "-std=c99", "-fsyntax-only", f"-I{INC}", "-I/usr/local/cuda/include", str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_go_float_format():
    """Table values are written as Go's fmt.Fprint writes float64 (table.go:45)."""
    from mumax2.engine import go_float
    assert [go_float(v) for v in [1e-11, 1.5e6, 0.25, -3.2e-5, 123456.0, 1.0, 0.0, 1e6, 2.5e-4]] == \
        ["1e-11", "1.5e+06", "0.25", "-3.2e-05", "123456", "1", "0", "1e+06", "0.00025"]
