"""The hand-written FFT against cuFFT.

The product never builds the real-space grid in HBM: spreading feeds the x
transform in shared memory (or the tcgen05 spread computes spread + x DFT as
one product), and the y and z transforms run as separate passes.  The
forward-spectrum diagnostic (sdt_spme_spectrum_device) runs that chain up to
the end of the forward z transform and returns the half spectra.  Here they
are compared with torch.fft.rfftn (cuFFT, FP64) of the spread grid built in
FP64 by the numpy oracle from the same particles and forces -- the grid the
reference spreads in src/mob/spme.cc:313-363 and transforms with MKL DFTI in
src/mob/spme.cc:754-756.

Bar: relative Frobenius error <= 1e-6 per component (FP32 spread and FFT)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _case(name, nrhs, seed):
    import torch
    import stokesdt_b200 as sdt
    from oracle import spme_oracle as so
    g = golden(name)
    N = len(g["rdi"])
    n3 = 3 * N
    K, p, L = int(g["K"]), int(g["p"]), float(g["box"])
    assert np.all(g["rdi"] == 1.0)
    m = sdt.MobSpme(N, g["rdi"], L, float(g["xi"]), float(g["rmax"]), K, p)
    assert m.Init(), m.last_error
    m.Update(g["pos"])
    F = np.random.default_rng(seed).standard_normal((nrhs, n3))
    dev = torch.device("cuda", 0)
    d_f = torch.tensor(F, device=dev)
    H1 = K // 2 + 1
    d_spec = torch.empty((nrhs, 3, K, K, H1), dtype=torch.complex64, device=dev)
    m.spectrum_device(nrhs, n3, d_f.data_ptr(), d_spec.data_ptr())
    torch.cuda.synchronize()
    spec = d_spec.cpu().numpy()
    o = so.SpmeOracle(g["rdi"], L, float(g["xi"]), float(g["rmax"]), K, p)
    o.update(g["pos"])
    for r in range(nrhs):
        grid = torch.tensor(o._spread(F[r].reshape(N, 3)), device=dev)   # [3][z][y][x] FP64
        ref = torch.fft.rfftn(grid, dim=(1, 2, 3)).cpu().numpy()          # cuFFT, FP64
        for c in range(3):
            # complex relative Frobenius error (real and imaginary parts)
            err = float(np.linalg.norm(ref[c] - spec[r, c]) / np.linalg.norm(ref[c]))
            assert err < TOL, (name, r, c, err)


def test_spectrum_k64_vs_cufft(gpu_available):
    """K = 64 (config 1 grid), 2 RHS: shared-memory spread + x FFT."""
    _case("spme_cfg1", 2, 11)


def test_spectrum_k256_shared_memory_spread_vs_cufft(gpu_available):
    """K = 256, 1 RHS: shared-memory spread + x FFT, TMA y pass, fused z pass."""
    _case("spme_N1000_K256_p6", 1, 12)


def test_spectrum_k256_tensor_core_spread_vs_cufft(gpu_available):
    """K = 256, 8 RHS: the tcgen05 spread + x DFT, then the same y and z passes."""
    _case("spme_N1000_K256_p6", 8, 13)
