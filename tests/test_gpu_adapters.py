"""GPU parity through the C++ adapters: the reference's own SPME and Lanczos
tests (tests/spme/testspme.cc:103-145, tests/lanczos/testlanczos.cc:81-148 of
the reference project) with MobSpmeGpu / BrwnLanczosGpu in place of MobSpme /
BrwnLanczos, called through the reference's MobBase / BrwnBase interfaces by
the compiled program tests/_bin/adapter_parity (tests/adapter_parity.cc,
built against the reference headers by tests/adapter_build.py).

Inputs and expected outputs are the committed golden vectors of the
reference's N1000_Phi0.1.xyz case: MobSpme and dense MobEwald products
(3 RHS, alpha 2.1, beta 1.1; bar 1e-6, and 1e-10 for MobEwaldGpu, FP64) and
the dense symmetric square root of the Ewald matrix applied to the Lanczos
vectors (bar 1e-5)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, golden, rel_err

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "tests", "_bin", "adapter_parity")


def _run(pos, rdi, box, K, p, xi, rmax, alpha, beta, tol, f, z):
    N = len(rdi)
    nr = f.shape[0]
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as fh:
            fh.write(np.array([N, nr, K, p], dtype=np.int32).tobytes())
            fh.write(np.array([box, xi, rmax, alpha, beta, tol], dtype=np.float64).tobytes())
            for a in (pos, rdi, f, z):
                fh.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        res = subprocess.run([EXE, fin, fout], capture_output=True, text=True, timeout=600)
        assert res.returncode == 0, res.stderr
        out = np.fromfile(fout, dtype=np.float64)
    n3 = 3 * N
    parts = np.split(out, np.cumsum([nr * n3] * 3 + [n3, nr * n3]))
    return {"v_full": parts[0].reshape(nr, n3), "v_real": parts[1].reshape(nr, n3),
            "v_recip": parts[2].reshape(nr, n3), "y1": parts[3], "y": parts[4].reshape(nr, n3),
            "v_ewald": parts[5].reshape(nr, n3)}


@pytest.mark.skipif(not os.access(EXE, os.X_OK), reason="adapter_parity not built (needs the reference headers)")
def test_reference_tests_through_cpp_adapters(gpu_available):
    g = golden("spme_N1000_K256_p6")
    gl = golden("lanczos_N1000")
    assert np.array_equal(g["pos"], gl["pos"])
    out = _run(g["pos"], g["rdi"], float(g["box"]), int(g["K"]), int(g["p"]), float(g["xi"]),
               float(g["rmax"]), float(g["alpha"]), float(g["beta"]), 1e-7, g["f"], gl["z"])
    # testspme.cc: SPME against the dense Ewald product, and against the
    # reference's own MobSpme on the same inputs
    assert rel_err(g["v_ewald"], out["v_full"]) < 1e-6
    # MobEwaldGpu through MobBase against the reference's MobEwald (FP64)
    assert rel_err(g["v_ewald"], out["v_ewald"]) < 1e-10
    for key in ("v_full", "v_real", "v_recip"):
        assert rel_err(g[key], out[key]) < 1e-6, key
    # testlanczos.cc: Lanczos against the dense symmetric square root, 1 and 3 RHS
    assert rel_err(gl["y_sqrt"][:1], out["y1"][None, :]) < 1e-5
    assert rel_err(gl["y_sqrt"], out["y"]) < 1e-5
