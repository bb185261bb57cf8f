"""include/trinity.h keeps trinity's C++ API: the reference's own driver
programs (src/main.cpp, examples/adapt.cpp) compile unchanged against it, and
the CLI built from it links to the in-tree library."""
import os
import subprocess

import pytest

from tests.oracle_lib import REF_SRC as REF

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")), reason="reference sources not mounted")
@pytest.mark.parametrize("src", ["src/main.cpp", "examples/adapt.cpp"])
def test_reference_drivers_compile_against_the_shim(src):
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I" + os.path.join(REPO, "include"),
                        '-DTRINITY_EXAMP_DIR="x"', '-DTRINITY_BUILD_DIR="y"', os.path.join(REF, src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]


def test_cli_is_built_and_prints_usage():
    exe = os.path.join(REPO, "trinity_b200", "bin", "trinity")
    assert os.path.exists(exe)
    r = subprocess.run([exe, "-h"], capture_output=True, text=True)
    assert r.returncode == 0 and "-i mesh -s solut" in r.stdout
    r = subprocess.run([exe, "-i", "/nonexistent.mesh", "-s", "x.bb"], capture_output=True, text=True)
    assert r.returncode != 0 and "invalid mesh file" in r.stdout
