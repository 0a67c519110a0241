"""The C binding a maintainer adds to the reference
(bh_ringdown_b200/integration/body_bhr.c, shown in INTEGRATION.md, in
place of HighOrder/body.cu and kern.cu) compiles as C and as C++ against
include/bhr.h and the reference's parm.h macros, and, built as the
reference's build.sh builds main.c and proj.c (g++), links against
libbhr.so.  tests/test_dropin.py runs the linked program on a GPU."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
from oracle.build_ref import default_reference_root  # noqa: E402

REF = default_reference_root()
HO = os.path.join(REF, "TD_GPU_code", "HighOrder")
LIB = os.path.join(ROOT, "bh_ringdown_b200", "libbhr.so")

# The macro names and values of HighOrder/parm.h that body_bhr.c reads, for
# when the reference tree is not present.
PARM_H = """#define N 16000
#define M 256
#define Xmax 50.0
#define Xmin -50.0
#define Text 90.0
#define Nd 100
#define Fr 50
#define T  1500.0
#define PTSX 128
#define PTSY 128
#define Pi 3.14159265358979
#define idx(b,a) (N*(b)+(a))
"""


SOURCE = os.path.join(ROOT, "bh_ringdown_b200", "integration", "body_bhr.c")


def example_source():
    return open(SOURCE).read()


def test_integration_doc_shows_the_committed_source():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"```c\n(/\* body_bhr\.c.*?)```", text, re.S)
    assert m, "INTEGRATION.md has no body_bhr.c block"
    assert m.group(1) == example_source()


@pytest.fixture
def workdir(tmp_path):
    (tmp_path / "body_bhr.c").write_text(example_source())
    parm = os.path.join(HO, "parm.h")
    if os.path.exists(parm):
        shutil.copy(parm, tmp_path / "parm.h")
    else:
        (tmp_path / "parm.h").write_text(PARM_H)
    return tmp_path


def run(cmd, cwd):
    out = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    assert out.returncode == 0, " ".join(cmd) + "\n" + out.stderr[-3000:]


@pytest.mark.parametrize("compiler", [["gcc", "-std=gnu11"], ["g++", "-std=c++17", "-x", "c++"]])
def test_example_compiles(workdir, compiler):
    run(compiler + ["-Wall", "-Werror", "-c", "body_bhr.c", "-I.", "-I" + os.path.join(ROOT, "include"),
                    "-o", "body_bhr.o"], workdir)


def test_example_links_with_the_reference_driver(workdir):
    if not os.path.exists(os.path.join(HO, "main.c")):
        pytest.skip("the reference tree is not present")
    if not os.path.exists(LIB):
        pytest.skip("libbhr.so is not built")
    run(["g++", "-O", "-c", os.path.join(HO, "main.c"), os.path.join(HO, "proj.c"), "-I."], workdir)
    run(["g++", "-O", "-c", "body_bhr.c", "-I.", "-I" + os.path.join(ROOT, "include")], workdir)
    run(["g++", "-o", "run", "main.o", "proj.o", "body_bhr.o", "-L" + os.path.dirname(LIB), "-lbhr", "-lm"], workdir)
    assert (workdir / "run").exists()
