"""The C++ forwarding class shown in INTEGRATION.md compiles against the
C ABI header as a maintainer would add it next to fluid_3d (syntax and type
check only; p_fatal_error is the reference's PGMG error hook, stubbed)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_forwarding_class_compiles(tmp_path):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"```cpp\n(.*?)```", text, re.S)
    assert m, "no C++ block in INTEGRATION.md"
    src = tmp_path / "gpu_fluid_3d.cc"
    src.write_text("static void p_fatal_error(const char *, int) {}\n" + m.group(1) +
                   "\nint main() { gpu_fluid_3d f(\"x.cfg\"); f.initialize(); f.set_dt(1e-3); f.init_iter(1);"
                   " return f.step_forward(0); }\n")
    r = subprocess.run(["g++", "-std=c++11", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
