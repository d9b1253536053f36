"""The MEX gateways compile (syntax check against a declarations-only mex.h;
MATLAB and Octave are not installed here)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("src", ["uvMatrixAssemblySSTREAM_mex.c", "SSTREAM2dNR2_mex.c", "uvhAssembly_mex.c",
                                 "SSTREAM_TransientImplicit_mex.c"])
def test_gateway_compiles(src):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "mex", "stub"),
                        "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "mex", src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
