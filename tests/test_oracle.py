"""CPU tests: the numpy FP64 oracle is pinned against the golden vectors that
the reference's own compiled code produced (tests/golden/make_golden.py), and
the reference's known-answer tests (SPME vs dense Ewald <= 1e-6,
tests/spme/testspme.cc:138-145; Lanczos vs dense sqrt <= 1e-6,
tests/lanczos/testlanczos.cc:144-148) are re-checked on those vectors."""
import numpy as np
import pytest

from conftest import golden, rel_err
from oracle import spme_oracle as so

SPME_CASES = ["spme_N1000_K64", "spme_N3", "spme_cfg1", "spme_N412_poly", "spme_N1000_K256_p6"]


def _oracle_from(g):
    o = so.SpmeOracle(g["rdi"], float(g["box"]), float(g["xi"]), float(g["rmax"]), int(g["K"]),
                      int(g["p"]))
    o.update(g["pos"])
    return o


@pytest.mark.parametrize("name", SPME_CASES)
def test_oracle_matches_reference_golden(name):
    g = golden(name)
    o = _oracle_from(g)
    a, b = float(g["alpha"]), float(g["beta"])
    nr = 1 if int(g["K"]) >= 256 else g["f"].shape[0]   # keep the CPU suite short
    f = g["f"][:nr]
    vr = o.mulvec(f, a, 0.0, mode="real")
    vk = o.mulvec(f, a, 0.0, mode="recip")
    for key, v in (("v_real", vr + b * f), ("v_recip", vk + b * f), ("v_full", vr + vk + b * f)):
        assert rel_err(g[key][:nr], v) < 1e-12, (name, key)


@pytest.mark.parametrize("name", ["spme_N1000_K256_p6", "spme_N1000_K256_p8", "spme_N412_poly",
                                  "spme_cfg1"])
def test_reference_known_answer_spme_vs_ewald(name):
    g = golden(name)
    assert rel_err(g["v_ewald"], g["v_full"]) < 1e-6


def test_reference_known_answer_lanczos():
    g = golden("lanczos_N1000")
    y0 = g["y_sqrt"]
    assert rel_err(y0[:1], g["y_ref1"]) < 1e-6
    assert rel_err(y0, g["y_ref3"]) < 1e-6


def test_oracle_lanczos_small_dense():
    """Oracle single and block Lanczos vs the dense symmetric square root of the
    oracle's own dense Ewald matrix (N = 40 particles of the N1000 geometry)."""
    g = golden("lanczos_N1000")
    pos = g["pos"][:40]
    M = so.dense_ewald_matrix(pos, np.ones(40), float(g["box"]), 1e-12)
    assert np.allclose(M, M.T)
    w, V = np.linalg.eigh(M)
    S = (V * np.sqrt(w)) @ V.T
    rng = np.random.default_rng(0)
    Z = rng.standard_normal((120, 4))
    y, it = so.lanczos_sqrt(lambda x: M @ x, Z[:, 0], 100, 1e-10)
    assert it > 0 and rel_err(S @ Z[:, 0], y) < 1e-8
    Y, itb = so.block_lanczos_sqrt(lambda X: M @ X, Z, 100, 1e-10)
    assert itb > 0 and rel_err(S @ Z, Y) < 1e-8


def test_oracle_block_of_one_is_single_vector_lanczos():
    """A block of one column is the single-vector recurrence
    (brwn_lanczos.cc:16-82 against :85-201 at k = 1): same stopping
    iteration, same iterate to rounding -- the identity the GPU's
    single-vector iteration relies on when it replaces the block QR by one
    normalisation."""
    g = golden("lanczos_N1000")
    pos = g["pos"][:40]
    M = so.dense_ewald_matrix(pos, np.ones(40), float(g["box"]), 1e-12)
    z = np.random.default_rng(4).standard_normal(120)
    for tol in (1e-5, 1e-8):
        y, it = so.lanczos_sqrt(lambda x: M @ x, z, 100, tol)
        Y, itb = so.block_lanczos_sqrt(lambda X: M @ X, z[:, None], 100, tol)
        assert it > 0 and it == itb
        assert rel_err(y, Y[:, 0]) < 1e-12


def test_bspline_weights_partition_of_unity():
    for p in (4, 6, 8):
        for frac in (0.0, 0.25, 0.5, 0.999):
            w = [so.bspline(p, x - frac)[0] for x in range(p)]
            assert abs(sum(w) - 1.0) < 1e-14


def test_device_weight_recurrence_matches_reference_bspline():
    """The order recurrence the CUDA k_prep kernel uses (M_p(x + 1 - frac),
    spme.cu spline_weights) restated in Python equals BSpline of spme.cc:38-68."""
    def device_weights(p, frac):
        t = 1.0 - frac
        w = [1.0] + [0.0] * (p - 1)
        for k in range(2, p + 1):
            for x in range(k - 1, -1, -1):
                cur = w[x] if x <= k - 2 else 0.0
                left = w[x - 1] if x >= 1 else 0.0
                w[x] = ((t + x) * cur + (k - t - x) * left) / (k - 1)
        return np.array(w)
    rng = np.random.default_rng(3)
    for p in (2, 4, 6, 8):
        for frac in list(rng.uniform(0, 1, 20)) + [0.0]:
            ref = np.array([so.bspline(p, x - frac)[0] for x in range(p)])
            assert np.max(np.abs(device_weights(p, frac) - ref)) < 1e-15


def test_xi_to_rmax_matches_survey_values():
    # XitoRmax(tol 1e-6) at L = 127.944 (ewald.cc:43-62)
    L = so.box_for(100000, 0.2)
    assert abs(so.xi_to_rmax(0.35, 1e-6, L) - 13.396) < 1e-3
    assert abs(so.xi_to_rmax(0.30, 1e-6, L) - 15.472) < 1e-3


def test_rsa_positions_non_overlapping():
    L = so.box_for(500, 0.3)
    pos = so.rsa_positions(500, L, 21)
    from scipy.spatial import cKDTree
    t = cKDTree(np.mod(pos, L), boxsize=L)
    assert len(t.query_pairs(2.0 - 1e-12)) == 0
    assert np.all((pos >= 0) & (pos < L))


@pytest.mark.parametrize("name", ["steric_N412_poly", "steric_cfg3"])
def test_steric_oracle_matches_reference_golden(name):
    """The numpy restatement of StericForce / PairListS reproduces the
    reference's own output (golden, made by the compiled reference)."""
    from oracle import spme_oracle as so
    g = golden(name)
    f = so.steric_force(g["pos"], g["rdi"], float(g["box"]), float(g["r0"]), float(g["k0"])) + g["f0"]
    assert np.linalg.norm(f - g["f"]) <= 1e-12 * np.linalg.norm(g["f"] - g["f0"])
