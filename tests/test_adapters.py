"""CPU test: the header-only C++ adapters (include/stokesdt_b200_adapters.hpp)
compile against the reference's own MobBase/BrwnBase/ForceBase headers in the
reference's C++ dialect (gnu++98) and link against libstokesdt_b200.so.
Skipped where the reference tree is absent (its headers are not vendored)."""
import os
import subprocess
import tempfile

import pytest

from conftest import ROOT

REF = os.environ.get("STOKESDT_REFERENCE", "/root/reference")

TU = r"""
#include "force_base.h"
#include "stokesdt_b200_adapters.hpp"
int main()
{
    double rdi[3] = {1.0, 1.0, 1.0};
    stokesdt::MobSpmeGpu m(3, rdi, 10.0, 0.5, 3.0, 32, 6);
    stokesdt::MobEwaldGpu ew(3, rdi, 10.0, 1e-12);
    if (ew.dim() != 9) return 1;
    stokesdt::BrwnLanczosGpu b(9, 10, 2, 1e-6);
    stokesdt::StericForceGpu s(3, rdi, 10.0, 2.0, 125.0);
    stokesdt::MobBase *base = &m;
    stokesdt::BrwnBase *bb = &b;
    stokesdt::ForceBase *fb = &s;
    (void)bb;
    (void)fb;
    return base->dim() == 9 ? 0 : 1;
}
"""


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src", "mob")), reason="reference tree absent")
def test_adapters_compile_link_and_run_against_reference_headers():
    import stokesdt_b200 as sdt
    import adapter_build
    sdt.lib()
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "tu.cc")
        exe = os.path.join(d, "tu")
        with open(src, "w") as fh:
            fh.write(TU)
        # MobBase/BrwnBase constructors and destructors live in the reference's .cc files
        cmd = adapter_build.compile_cmd(REF, src, exe)
        cmd[-1] = "-Wl,-rpath," + os.path.join(ROOT, "stokesdt_b200")
        res = subprocess.run(cmd, capture_output=True, text=True)
        assert res.returncode == 0, res.stderr
        assert subprocess.run([exe]).returncode == 0


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src", "mob")), reason="reference tree absent")
def test_adapter_parity_program_builds():
    """The program the GPU adapter test runs (tests/adapter_parity.cc), built
    against the reference headers into tests/_bin/ (it travels prebuilt)."""
    import stokesdt_b200 as sdt
    import adapter_build
    sdt.lib()
    exe = adapter_build.build(REF)
    assert os.access(exe, os.X_OK)
