"""GPU test of sdt_spme_real_mulvec_noalloc, the real-space product for
callers that may not allocate device memory (fixed-budget runtimes, code that
owns every allocation): it must give what the allocating entry point
sdt_spme_mulvec_device(SDT_MOB_REAL) gives, on two calls in a row (the
shared scratch array keeps the first call's contents), and refuse sizes
beyond its fixed array.  This file sorts last so a stop-at-first-failure run
has run every other test before it."""
import ctypes

import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-6


def test_noalloc_real_product_matches_allocating_entry_point(gpu_available):
    import torch
    import stokesdt_b200 as sdt
    L = sdt.lib()
    g = golden("spme_cfg1")
    N = len(g["rdi"])
    n3 = 3 * N
    m = sdt.MobSpme(N, g["rdi"], float(g["box"]), float(g["xi"]), float(g["rmax"]), 64, 6)
    assert m.Init()
    m.Update(g["pos"])
    rng = np.random.default_rng(17)
    for call, (nr, alpha, beta) in enumerate(((4, 1.3, 0.0), (16, -0.7, 1.1))):
        f = torch.tensor(rng.standard_normal((nr, n3)), device="cuda")
        v0 = torch.tensor(rng.standard_normal((nr, n3)), device="cuda")
        v_ref = v0.clone()
        v_new = v0.clone()
        m.mulvec_device(sdt.MODE_REAL, nr, alpha, n3, f.data_ptr(), beta, n3, v_ref.data_ptr())
        st = L.sdt_spme_real_mulvec_noalloc(m.handle, nr, alpha, n3, ctypes.c_void_p(f.data_ptr()),
                                            beta, n3, ctypes.c_void_p(v_new.data_ptr()))
        assert st == 0, L.sdt_spme_last_error(m.handle)
        m.synchronize()
        err = rel_err(v_ref.cpu().numpy(), v_new.cpu().numpy())
        assert err < TOL, (call, err)


def test_noalloc_rejects_sizes_beyond_its_array(gpu_available):
    import torch
    import stokesdt_b200 as sdt
    L = sdt.lib()
    N = 20000
    box = 60.0
    pos = np.random.default_rng(0).uniform(0, box, (N, 3))
    m = sdt.MobSpme(N, np.ones(N), box, 0.5, 8.0, 64, 6)
    assert m.Init()
    m.Update(pos)
    nr = 14      # 20000 * 14 = 280000 > 262144
    f = torch.zeros((nr, 3 * N), dtype=torch.float64, device="cuda")
    v = torch.zeros_like(f)
    st = L.sdt_spme_real_mulvec_noalloc(m.handle, nr, 1.0, 3 * N, ctypes.c_void_p(f.data_ptr()), 0.0,
                                        3 * N, ctypes.c_void_p(v.data_ptr()))
    assert st == -1
    assert b"262144" in L.sdt_spme_last_error(m.handle)


def _noalloc(L, m, nr, alpha, ldf, f, beta, ldv, v):
    st = L.sdt_spme_real_mulvec_noalloc(m.handle, nr, alpha, ldf, ctypes.c_void_p(f.data_ptr()), beta, ldv,
                                        ctypes.c_void_p(v.data_ptr()))
    assert st == 0, L.sdt_spme_last_error(m.handle)


def test_noalloc_allocates_nothing_on_a_fresh_engine(gpu_available):
    """On an engine that has never run a product (so it holds no product work
    buffers), the first call leaves the device's free memory unchanged.  A
    first call on another engine comes before, so the library's module is
    loaded and the array's address looked up outside the measured call."""
    import torch
    import stokesdt_b200 as sdt
    L = sdt.lib()
    g = golden("spme_cfg1")
    N = len(g["rdi"])
    n3 = 3 * N
    args = (N, g["rdi"], float(g["box"]), float(g["xi"]), float(g["rmax"]), 64, 6)
    warm = sdt.MobSpme(*args)
    assert warm.Init()
    warm.Update(g["pos"])
    f = torch.tensor(np.random.default_rng(3).standard_normal((2, n3)), device="cuda")
    v = torch.zeros_like(f)
    _noalloc(L, warm, 2, 1.0, n3, f, 0.0, n3, v)
    warm.synchronize()
    m = sdt.MobSpme(*args)
    assert m.Init()
    m.Update(g["pos"])
    v_new = torch.zeros_like(f)
    m.synchronize()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    _noalloc(L, m, 2, 1.0, n3, f, 0.0, n3, v_new)
    m.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, (free0, free1)
    v_ref = torch.zeros_like(f)
    m.mulvec_device(sdt.MODE_REAL, 2, 1.0, n3, f.data_ptr(), 0.0, n3, v_ref.data_ptr())
    m.synchronize()
    assert rel_err(v_ref.cpu().numpy(), v_new.cpu().numpy()) < TOL


def test_noalloc_padded_leading_dimensions_and_in_place(gpu_available):
    """ldf = ldv = 3N + 8 with beta != 0, against the allocating product on the
    same padded buffers; then the same call in place (d_f == d_v)."""
    import torch
    import stokesdt_b200 as sdt
    L = sdt.lib()
    g = golden("spme_cfg1")
    N = len(g["rdi"])
    n3 = 3 * N
    ld = n3 + 8
    m = sdt.MobSpme(N, g["rdi"], float(g["box"]), float(g["xi"]), float(g["rmax"]), 64, 6)
    assert m.Init()
    m.Update(g["pos"])
    rng = np.random.default_rng(29)
    nr, alpha, beta = 3, 0.9, -0.4
    f = torch.tensor(rng.standard_normal(nr * ld), device="cuda")
    v0 = torch.tensor(rng.standard_normal(nr * ld), device="cuda")
    v_ref, v_new = v0.clone(), v0.clone()
    m.mulvec_device(sdt.MODE_REAL, nr, alpha, ld, f.data_ptr(), beta, ld, v_ref.data_ptr())
    _noalloc(L, m, nr, alpha, ld, f, beta, ld, v_new)
    m.synchronize()
    ref = v_ref.cpu().numpy().reshape(nr, ld)
    new = v_new.cpu().numpy().reshape(nr, ld)
    assert rel_err(ref[:, :n3], new[:, :n3]) < TOL
    # the padding between vectors is left alone
    assert np.array_equal(new[:, n3:], v0.cpu().numpy().reshape(nr, ld)[:, n3:])
    # in place: v := alpha M_real v + beta v
    w_ref, w_new = f.clone(), f.clone()
    tmp = f.clone()
    m.mulvec_device(sdt.MODE_REAL, nr, alpha, ld, tmp.data_ptr(), beta, ld, w_ref.data_ptr())
    _noalloc(L, m, nr, alpha, ld, w_new, beta, ld, w_new)
    m.synchronize()
    a = w_ref.cpu().numpy().reshape(nr, ld)[:, :n3]
    b = w_new.cpu().numpy().reshape(nr, ld)[:, :n3]
    assert rel_err(a, b) < TOL
