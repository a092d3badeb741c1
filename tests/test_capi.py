"""The C-ABI library: it builds, loads, exports every declared entry point, its
struct layout matches the ctypes mirror, and its host-only functions work.
No compute calls that need a GPU.  CPU only."""
import ctypes as C
import re
import subprocess
import textwrap
from pathlib import Path

import numpy as np
import pytest

from oracle import rigw_oracle as o

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "rigw.h"


@pytest.fixture(scope="module")
def lib():
    from molgw_b200 import build
    build.build()
    from molgw_b200 import rigw
    return rigw.load_library()


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"RIGW_API\s+[\w\s\*]+?\b(rigw_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported(lib):
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s
    out = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "molgw_b200" / "librigw.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (rigw_\w+)", out))
    assert set(syms) <= exported
    # nothing beyond the C ABI leaks out of the library
    assert exported == set(syms)


def test_struct_layout_matches_ctypes(tmp_path):
    from molgw_b200.rigw import Problem, Result
    src = tmp_path / "layout.c"
    fields_p = [f for f, _ in Problem._fields_]
    fields_r = [f for f, _ in Result._fields_]
    body = "".join(f'  printf("P {f} %zu\\n", offsetof(rigw_problem, {f}));\n' for f in fields_p)
    body += "".join(f'  printf("R {f} %zu\\n", offsetof(rigw_result, {f}));\n' for f in fields_r)
    src.write_text(textwrap.dedent(f"""
        #include <stdio.h>
        #include <stddef.h>
        #include "rigw.h"
        int main(void) {{
          printf("SP %zu\\nSR %zu\\n", sizeof(rigw_problem), sizeof(rigw_result));
        {body}  return 0;
        }}
    """))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    vals = {}
    for line in out:
        if line:
            parts = line.split()
            vals[tuple(parts[:-1])] = int(parts[-1])
    assert vals[("SP",)] == C.sizeof(Problem)
    assert vals[("SR",)] == C.sizeof(Result)
    for f in fields_p:
        assert vals[("P", f)] == getattr(Problem, f).offset, f
    for f in fields_r:
        assert vals[("R", f)] == getattr(Result, f).offset, f


def test_constants_match_the_header(tmp_path):
    """Precision codes, techniques, problem flags and status codes of the Python
    mirror are the header's values."""
    from molgw_b200 import rigw
    names = ["RIGW_FP64", "RIGW_BF16X3", "RIGW_OZAKI_INT8", "RIGW_PADE", "RIGW_HOMOLUMO",
             "RIGW_PROBLEM_DEVICE_POINTERS", "RIGW_PROBLEM_QP_ONLY", "RIGW_PROBLEM_SPIN_CHANNEL"]
    src = tmp_path / "consts.c"
    body = "".join(f'  printf("{n} %d\\n", (int){n});\n' for n in names)
    src.write_text("#include <stdio.h>\n#include \"rigw.h\"\nint main(void) {\n" + body + "  return 0;\n}\n")
    exe = tmp_path / "consts"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    vals = dict(zip(out[0::2], map(int, out[1::2])))
    for n in names:
        assert vals[n] == getattr(rigw, n), n
    assert rigw.RIGW_OZAKI(5) == vals["RIGW_OZAKI_INT8"] + 5


def test_imag_grid_matches_oracle(lib):
    from molgw_b200 import rigw
    for n in (1, 16, 32, 48, 64):
        om, wt = rigw.imag_grid(n)
        om_o, wt_o = o.imaginary_quad_grid(n)
        assert np.allclose(om, om_o, rtol=1e-14, atol=0)
        assert np.allclose(wt, wt_o, rtol=1e-14, atol=0)


def test_bad_arguments_return_status_not_abort(lib):
    assert lib.rigw_imag_grid(0, None, None) == 1
    assert lib.rigw_create(None, 0, 0) == 1
    assert lib.rigw_g0w0(None, None, None) == 1
    assert lib.rigw_sox_selfenergy_imag(None, None, None) == 1
    assert lib.rigw_sosex_selfenergy_imag(None, None, None, None) == 1
    assert lib.rigw_version() == 1


def test_footprint_grows_with_size(lib):
    a = lib.rigw_footprint_bytes(840, 21, 207, 32, 228, 2, 0)
    b = lib.rigw_footprint_bytes(4000, 100, 1100, 48, 1200, 2, 0)
    # eps + rhs dominate: 32 * 896^2 * 8 B ~ 205 MB at the 840-function size
    assert 2e8 < a < 2e9 and b > 10 * a


def test_no_cpu_fallback_without_device(lib):
    """Without a CUDA device the engine refuses to start (there is no CPU path)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from molgw_b200.rigw import Engine, RigwError
    with pytest.raises(RigwError):
        Engine(0)


def test_tune_report_layout_matches_ctypes(tmp_path):
    from molgw_b200.rigw import TuneReport
    fields = [f for f, _ in TuneReport._fields_]
    body = "".join(f'  printf("T {f} %zu\\n", offsetof(rigw_tune_report, {f}));\n' for f in fields)
    src = tmp_path / "tune.c"
    src.write_text(textwrap.dedent(f"""
        #include <stdio.h>
        #include <stddef.h>
        #include "rigw.h"
        int main(void) {{
          printf("S %zu\\n", sizeof(rigw_tune_report));
        {body}  return 0;
        }}
    """))
    exe = tmp_path / "tune"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in
               subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n") if line)
    assert int(out["S"]) == C.sizeof(TuneReport)
    for f in fields:
        assert int(out[f"T {f}"]) == getattr(TuneReport, f).offset, f


def test_sox_problem_layout_matches_ctypes(tmp_path):
    from molgw_b200.rigw import SoxProblem
    fields = [f for f, _ in SoxProblem._fields_]
    body = "".join(f'  printf("X {f} %zu\\n", offsetof(rigw_sox_problem, {f}));\n' for f in fields)
    src = tmp_path / "sox.c"
    src.write_text(textwrap.dedent(f"""
        #include <stdio.h>
        #include <stddef.h>
        #include "rigw.h"
        int main(void) {{
          printf("S %zu\\n", sizeof(rigw_sox_problem));
        {body}  return 0;
        }}
    """))
    exe = tmp_path / "sox"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in
               subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n") if line)
    assert int(out["S"]) == C.sizeof(SoxProblem)
    for f in fields:
        assert int(out[f"X {f}"]) == getattr(SoxProblem, f).offset, f


def test_sosex_problem_layout_matches_ctypes(tmp_path):
    from molgw_b200.rigw import SosexProblem
    fields = [f for f, _ in SosexProblem._fields_]
    body = "".join(f'  printf("X {f} %zu\\n", offsetof(rigw_sosex_problem, {f}));\n' for f in fields)
    src = tmp_path / "sosex.c"
    src.write_text(textwrap.dedent(f"""
        #include <stdio.h>
        #include <stddef.h>
        #include "rigw.h"
        int main(void) {{
          printf("S %zu\\n", sizeof(rigw_sosex_problem));
        {body}  return 0;
        }}
    """))
    exe = tmp_path / "sosex"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in
               subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n") if line)
    assert int(out["S"]) == C.sizeof(SosexProblem)
    for f in fields:
        assert int(out[f"X {f}"]) == getattr(SosexProblem, f).offset, f


@pytest.mark.parametrize("cname,pyname", [("rigw_contour_problem", "ContourProblem"), ("rigw_dm_problem", "DmProblem"),
                                          ("rigw_shell", "RiShell"), ("rigw_ri_problem", "RiProblem"),
                                          ("rigw_contour_result", "ContourResult")])
def test_contour_layouts_match_ctypes(tmp_path, cname, pyname):
    from molgw_b200 import rigw
    cls = getattr(rigw, pyname)
    fields = [f for f, _ in cls._fields_]
    body = "".join(f'  printf("X {f} %zu\\n", offsetof({cname}, {f}));\n' for f in fields)
    src = tmp_path / "contour.c"
    src.write_text(textwrap.dedent(f"""
        #include <stdio.h>
        #include <stddef.h>
        #include "rigw.h"
        int main(void) {{
          printf("S %zu\\n", sizeof({cname}));
        {body}  return 0;
        }}
    """))
    exe = tmp_path / "contour"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in
               subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n") if line)
    assert int(out["S"]) == C.sizeof(cls)
    for f in fields:
        assert int(out[f"X {f}"]) == getattr(cls, f).offset, f
