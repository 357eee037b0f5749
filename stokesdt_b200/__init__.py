"""stokesdt_b200 -- B200-native SPME Rotne-Prager-Yamakawa mobility product and
block-Lanczos Brownian displacement, behind StokesDT's own interfaces.

Host-side mirror of the reference's operator interface for this path
(paths relative to the StokesDT project):

  MobSpme(npos, rdi, box_size, xi, rmax, dim, porder)      src/mob/mob_spme.h:27-33
      .Init() -> bool                                       src/mob/mob_spme.cc:53-132
      .Update(pos, rdi)                                     src/mob/mob_spme.cc:205-216
      .MulVector(num_rhs, alpha, ldf, f, beta, ldv, v)      src/mob/mob_spme.cc:219-236
      .RealMulVector(...), .RecipMulVector(...)             src/mob/mob_spme.cc:239-263
      .dim()                                                src/mob/mob_spme.h:94
  BrwnLanczos(dim, max_iters, max_nrhs, tol)                src/brwn/brwn_lanczos.h:44-45
      .Init() -> bool                                       src/brwn/brwn_lanczos.cc:224-275
      .Compute(mob, num_rhs, ldz, z, ldy, y)                src/brwn/brwn_lanczos.cc:278-304

Vectors are numpy float64 arrays laid out like the reference's C arrays: a
block of ``num_rhs`` vectors of leading dimension ``ld`` is a flat array (or a
``(num_rhs, ld)`` array) with vector j at offset ``j*ld``; particle i's
component c is element ``3*i + c``.  Every call goes through the C ABI of the
in-tree CUDA library ``libstokesdt_b200.so`` (``include/stokesdt_b200.h``);
there is no CPU fallback -- importing works without a GPU, but creating an
engine on a machine without one raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = ["MobSpme", "MobEwald", "BrwnLanczos", "lib", "LIB_PATH", "StokesError", "MODE_FULL", "MODE_REAL",
           "MODE_RECIP"]

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libstokesdt_b200.so")

MODE_FULL, MODE_REAL, MODE_RECIP = 0, 1, 2
STATUS = {0: "SDT_OK", -1: "SDT_ERR_INVALID", -2: "SDT_ERR_CUDA", -3: "SDT_ERR_ALLOC",
          -4: "SDT_ERR_STATE", -5: "SDT_ERR_NOT_CONVERGED", -6: "SDT_ERR_UNSUPPORTED"}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_lib = None

# Every symbol include/stokesdt_b200.h declares, with its ctypes signature.
SIGNATURES = {
    "sdt_version": (ctypes.c_char_p, []),
    "sdt_spme_create": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(_vp)]),
    "sdt_spme_update": (ctypes.c_int, [_vp, _dp]),
    "sdt_spme_update_device": (ctypes.c_int, [_vp, _vp]),
    "sdt_spme_mulvec": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_int, _dp, ctypes.c_double, ctypes.c_int, _dp]),
    "sdt_spme_mulvec_device": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                              ctypes.c_int, _vp, ctypes.c_double, ctypes.c_int,
                                              _vp]),
    "sdt_spme_real_mulvec_noalloc": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                    _vp, ctypes.c_double, ctypes.c_int, _vp]),
    "sdt_spme_dim": (ctypes.c_int, [_vp]),
    "sdt_spme_set_stream": (ctypes.c_int, [_vp, _vp]),
    "sdt_spme_set_pairlist": (ctypes.c_int, [_vp, ctypes.c_int]),
    "sdt_spme_pairlist_size": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "sdt_spme_synchronize": (ctypes.c_int, [_vp]),
    "sdt_bd_create": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.c_ulonglong,
                                     ctypes.POINTER(_vp)]),
    "sdt_bd_create_ewald": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.c_ulonglong,
                                           ctypes.POINTER(_vp)]),
    "sdt_bd_set_positions": (ctypes.c_int, [_vp, _dp]),
    "sdt_bd_get_positions": (ctypes.c_int, [_vp, _dp]),
    "sdt_bd_set_step": (ctypes.c_int, [_vp, ctypes.c_longlong]),
    "sdt_bd_advance": (ctypes.c_int, [_vp, ctypes.c_int]),
    "sdt_bd_info": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                   _ip]),
    "sdt_bd_draw_gaussian": (ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, _dp]),
    "sdt_bd_set_stream": (ctypes.c_int, [_vp, _vp]),
    "sdt_bd_synchronize": (ctypes.c_int, [_vp]),
    "sdt_bd_last_error": (ctypes.c_char_p, [_vp]),
    "sdt_bd_destroy": (None, [_vp]),
    "sdt_batch_create": (ctypes.c_int, [ctypes.c_int, _ip, _dp, _dp, _ip, _dp, _dp, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]),
    "sdt_batch_update_device": (ctypes.c_int, [_vp, _vp]),
    "sdt_batch_mulvec_device": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, _vp, ctypes.c_double,
                                               _vp]),
    "sdt_batch_lanczos_device": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _ip]),
    "sdt_batch_update": (ctypes.c_int, [_vp, _dp]),
    "sdt_batch_mulvec": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, _dp, ctypes.c_double, _dp]),
    "sdt_batch_lanczos": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp, _ip]),
    "sdt_batch_info": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong), _ip]),
    "sdt_batch_synchronize": (ctypes.c_int, [_vp]),
    "sdt_batch_set_packed": (ctypes.c_int, [_vp, ctypes.c_int]),
    "sdt_ewald_create": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_int, ctypes.POINTER(_vp)]),
    "sdt_ewald_update": (ctypes.c_int, [_vp, _dp]),
    "sdt_ewald_update_device": (ctypes.c_int, [_vp, _vp]),
    "sdt_ewald_mulvec": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, ctypes.c_double,
                                        ctypes.c_int, _dp]),
    "sdt_ewald_mulvec_device": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, _vp,
                                               ctypes.c_double, ctypes.c_int, _vp]),
    "sdt_ewald_get_matrix": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "sdt_ewald_info": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double), _ip, _ip]),
    "sdt_ewald_dim": (ctypes.c_int, [_vp]),
    "sdt_ewald_set_stream": (ctypes.c_int, [_vp, _vp]),
    "sdt_ewald_last_error": (ctypes.c_char_p, [_vp]),
    "sdt_ewald_destroy": (None, [_vp]),
    "sdt_lanczos_compute_ewald": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp,
                                                 _ip]),
    "sdt_lanczos_compute_ewald_device": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int,
                                                        _vp, _ip]),
    "sdt_batch_get_packed": (ctypes.c_int, [_vp]),
    "sdt_batch_last_error": (ctypes.c_char_p, [_vp]),
    "sdt_batch_destroy": (None, [_vp]),
    "sdt_serve_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.POINTER(_vp)]),
    "sdt_serve_register": (ctypes.c_int, [_vp, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp, _ip]),
    "sdt_serve_submit": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp,
                                        ctypes.POINTER(ctypes.c_longlong)]),
    "sdt_serve_wait": (ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]),
    "sdt_serve_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                       ctypes.POINTER(ctypes.c_double)]),
    "sdt_serve_last_error": (ctypes.c_char_p, [_vp]),
    "sdt_serve_batch_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong),
                                             ctypes.POINTER(ctypes.c_longlong), _ip]),
    "sdt_serve_destroy": (None, [_vp]),
    "sdt_xyz_count": (ctypes.c_int, [ctypes.c_char_p, _ip]),
    "sdt_xyz_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, _dp, _dp, _dp, _ip,
                                    ctypes.POINTER(ctypes.c_double)]),
    "sdt_xyz_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int,
                                     ctypes.c_double, _dp]),
    "sdt_config_get": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]),
    "sdt_model_steric": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_double)]),
    "sdt_steric_create": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.POINTER(_vp)]),
    "sdt_steric_accumulate": (ctypes.c_int, [_vp, _dp, _dp]),
    "sdt_steric_accumulate_device": (ctypes.c_int, [_vp, _vp, _vp]),
    "sdt_steric_set_stream": (ctypes.c_int, [_vp, _vp]),
    "sdt_steric_last_error": (ctypes.c_char_p, [_vp]),
    "sdt_steric_destroy": (None, [_vp]),
    "sdt_spme_last_error": (ctypes.c_char_p, [_vp]),
    "sdt_spme_destroy": (None, [_vp]),
    "sdt_lanczos_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_int, ctypes.POINTER(_vp)]),
    "sdt_lanczos_compute": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _dp,
                                           ctypes.c_int, _dp, _ip]),
    "sdt_lanczos_compute_device": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp,
                                                  ctypes.c_int, _vp, _ip]),
    "sdt_lanczos_set_reorth": (ctypes.c_int, [_vp, ctypes.c_int]),
    "sdt_lanczos_set_stream": (ctypes.c_int, [_vp, _vp]),
    "sdt_spme_profile_mulvec": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int]),
    "sdt_profile_stage_name": (ctypes.c_char_p, [ctypes.c_int]),
    "sdt_spme_spectrum_device": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "sdt_kernel_launches": (ctypes.c_ulonglong, []),
    "sdt_lanczos_history": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
    "sdt_lanczos_products": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "sdt_lanczos_last_error": (ctypes.c_char_p, [_vp]),
    "sdt_lanczos_destroy": (None, [_vp]),
}


class StokesError(RuntimeError):
    """A C-ABI call returned a negative sdt_status."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def lib():
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m stokesdt_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def kernel_launches() -> int:
    """Kernels launched by the library since it was loaded."""
    return int(lib().sdt_kernel_launches())


def _f64(a) -> np.ndarray:
    a = np.asarray(a, dtype=np.float64)
    if not a.flags["C_CONTIGUOUS"]:
        a = np.ascontiguousarray(a)
    return a


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class MobSpme:
    """SPME RPY mobility on one GPU (drop-in for the reference's MobSpme)."""

    def __init__(self, npos, rdi, box_size, xi, rmax, dim, porder, device=0):
        self.npos = int(npos)
        self.rdi = _f64(rdi).reshape(-1).copy()
        if self.rdi.size != self.npos:
            raise ValueError("rdi must have npos entries")
        self.box_size = float(box_size)
        self.xi = float(xi)
        self.rmax = float(rmax)
        self.dim_fft = int(dim)
        self.porder = int(porder)
        self.device = int(device)
        self._h = None
        self.last_error = ""

    # MobBase::Init
    def Init(self) -> bool:
        h = _vp()
        st = lib().sdt_spme_create(self.npos, _ptr(self.rdi), self.box_size, self.xi, self.rmax,
                                   self.dim_fft, self.porder, self.device, ctypes.byref(h))
        if st != 0:
            self.last_error = STATUS.get(st, str(st))
            return False
        self._h = h
        return True

    def _check(self, st):
        if st != 0:
            msg = lib().sdt_spme_last_error(self._h).decode() if self._h else ""
            raise StokesError(st, msg)

    def _need(self):
        if self._h is None:
            raise StokesError(-4, "Init() has not succeeded")

    # MobBase::Update (rdi is fixed at construction, as MobSpme copies it)
    def Update(self, pos, rdi=None):
        self._need()
        pos = _f64(pos).reshape(-1)
        if pos.size < 3 * self.npos:
            raise ValueError("pos must hold 3*npos values")
        self._check(lib().sdt_spme_update(self._h, _ptr(pos)))

    def _mul(self, mode, num_rhs, alpha, ldf, f, beta, ldv, v):
        self._need()
        f = _f64(f)
        if not isinstance(v, np.ndarray) or v.dtype != np.float64 or not v.flags["C_CONTIGUOUS"]:
            raise TypeError("v must be a C-contiguous float64 numpy array (updated in place)")
        if f.size < (num_rhs - 1) * ldf + 3 * self.npos or v.size < (num_rhs - 1) * ldv + 3 * self.npos:
            raise ValueError("f or v too small for num_rhs and the leading dimensions")
        self._check(lib().sdt_spme_mulvec(self._h, mode, int(num_rhs), float(alpha), int(ldf),
                                          _ptr(f), float(beta), int(ldv), _ptr(v)))

    def MulVector(self, num_rhs, alpha, ldf, f, beta, ldv, v):
        """v := alpha*M*f + beta*v (in place on v)."""
        self._mul(MODE_FULL, num_rhs, alpha, ldf, f, beta, ldv, v)

    def RealMulVector(self, num_rhs, alpha, ldf, f, beta, ldv, v):
        self._mul(MODE_REAL, num_rhs, alpha, ldf, f, beta, ldv, v)

    def RecipMulVector(self, num_rhs, alpha, ldf, f, beta, ldv, v):
        self._mul(MODE_RECIP, num_rhs, alpha, ldf, f, beta, ldv, v)

    # device-pointer variants (e.g. torch tensors' data_ptr()), asynchronous
    def update_device(self, d_pos: int):
        self._need()
        self._check(lib().sdt_spme_update_device(self._h, _vp(d_pos)))

    def mulvec_device(self, mode, num_rhs, alpha, ldf, d_f: int, beta, ldv, d_v: int):
        self._need()
        self._check(lib().sdt_spme_mulvec_device(self._h, mode, int(num_rhs), float(alpha), int(ldf),
                                                 _vp(d_f), float(beta), int(ldv), _vp(d_v)))

    def set_stream(self, stream_handle: int):
        self._need()
        self._check(lib().sdt_spme_set_stream(self._h, _vp(stream_handle)))

    def profile(self, num_rhs: int = 16, reps: int = 3) -> dict:
        """Mean milliseconds per stage of a num_rhs-vector product."""
        self._need()
        out = (ctypes.c_double * 16)()
        n = lib().sdt_spme_profile_mulvec(self._h, int(num_rhs), int(reps), out, 16)
        if n < 0:
            self._check(n)
        return {lib().sdt_profile_stage_name(i).decode(): out[i] for i in range(n)}

    def spectrum_device(self, num_rhs, ldf, d_f: int, d_spec: int):
        """Half spectra of the spread forces (forward transform only), written
        to d_spec as complex64 [num_rhs][3][K][K][K/2+1]; a diagnostic for
        checking the hand-written FFT against an independent one."""
        self._need()
        self._check(lib().sdt_spme_spectrum_device(self._h, int(num_rhs), int(ldf), _vp(d_f), _vp(d_spec)))

    def set_pairlist(self, enable: bool):
        """Store the real-space pairs at every Update (default) or walk the
        cell list inside every product; applies from the next Update."""
        self._need()
        self._check(lib().sdt_spme_set_pairlist(self._h, 1 if enable else 0))

    def pairlist_size(self) -> int:
        """Pairs in the current real-space pair list, -1 if none is used."""
        self._need()
        out = ctypes.c_longlong(0)
        self._check(lib().sdt_spme_pairlist_size(self._h, ctypes.byref(out)))
        return int(out.value)

    def synchronize(self):
        self._need()
        self._check(lib().sdt_spme_synchronize(self._h))

    def dim(self) -> int:
        return 3 * self.npos

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h is not None:
            lib().sdt_spme_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MobEwald:
    """Dense Ewald RPY mobility matrix on one GPU, FP64 (drop-in for the
    reference's MobEwald, src/mob/mob_ewald.h: Init / Update / MulVector /
    GetMatrix / dim).  xi = None selects the reference's default
    10^(1/6) sqrt(pi) / L."""

    def __init__(self, npos, rdi, box_size, tol, xi=None, device=0):
        self.npos = int(npos)
        self.rdi = _f64(rdi).reshape(-1).copy()
        if self.rdi.size != self.npos:
            raise ValueError("rdi must have npos entries")
        self.box_size = float(box_size)
        self.tol = float(tol)
        self.xi = 0.0 if xi is None else float(xi)
        self.device = int(device)
        self._h = None
        self.last_error = ""

    def Init(self) -> bool:
        h = _vp()
        st = lib().sdt_ewald_create(self.npos, _ptr(self.rdi), self.box_size, self.tol, self.xi, self.device,
                                    ctypes.byref(h))
        if st != 0:
            self.last_error = STATUS.get(st, str(st))
            return False
        self._h = h
        return True

    def _check(self, st):
        if st != 0:
            msg = lib().sdt_ewald_last_error(self._h).decode() if self._h else ""
            raise StokesError(st, msg)

    def _need(self):
        if self._h is None:
            raise StokesError(-4, "Init() has not succeeded")

    def Update(self, pos, rdi=None):
        self._need()
        pos = _f64(pos).reshape(-1)
        if pos.size < 3 * self.npos:
            raise ValueError("pos must hold 3*npos values")
        self._check(lib().sdt_ewald_update(self._h, _ptr(pos)))

    def MulVector(self, num_rhs, alpha, ldf, f, beta, ldv, v):
        """v := alpha*M*f + beta*v (in place on v)."""
        self._need()
        f = _f64(f)
        if not isinstance(v, np.ndarray) or v.dtype != np.float64 or not v.flags["C_CONTIGUOUS"]:
            raise TypeError("v must be a C-contiguous float64 numpy array (updated in place)")
        self._check(lib().sdt_ewald_mulvec(self._h, int(num_rhs), float(alpha), int(ldf), _ptr(f), float(beta),
                                           int(ldv), _ptr(v)))

    def GetMatrix(self):
        self._need()
        n = 3 * self.npos
        m = np.zeros((n, n))
        self._check(lib().sdt_ewald_get_matrix(self._h, n, _ptr(m)))
        return m

    def info(self) -> dict:
        xi, rmax, kmax = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        nr, nk = ctypes.c_int(), ctypes.c_int()
        self._check(lib().sdt_ewald_info(self._h, ctypes.byref(xi), ctypes.byref(rmax), ctypes.byref(kmax),
                                         ctypes.byref(nr), ctypes.byref(nk)))
        return {"xi": xi.value, "rmax": rmax.value, "kmax": kmax.value, "nimages": nr.value, "nk": nk.value}

    def dim(self) -> int:
        return 3 * self.npos

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h is not None:
            lib().sdt_ewald_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class StericForce:
    """Steric force on one GPU (drop-in for the reference's StericForce,
    src/force/force_steric.h: ForceBase::Init / Accumulate / Compute)."""

    def __init__(self, npos, rdi, box_size, steric_r0, steric_k0, device=0):
        self.npos = int(npos)
        self.rdi = _f64(rdi).reshape(-1).copy()
        if self.rdi.size != self.npos:
            raise ValueError("rdi must have npos entries")
        self.box_size = float(box_size)
        self.r0 = float(steric_r0)
        self.k0 = float(steric_k0)
        self.device = int(device)
        self._h = None
        self.last_error = ""

    def Init(self) -> bool:
        h = _vp()
        st = lib().sdt_steric_create(self.npos, _ptr(self.rdi), self.box_size, self.r0, self.k0,
                                     self.device, ctypes.byref(h))
        if st != 0:
            self.last_error = STATUS.get(st, str(st))
            return False
        self._h = h
        return True

    def _check(self, st):
        if st != 0:
            msg = lib().sdt_steric_last_error(self._h).decode() if self._h else ""
            raise StokesError(st, msg)

    def Accumulate(self, pos, rdi, f):
        """f += steric force at pos (f is updated in place and returned)."""
        if self._h is None:
            raise StokesError(-4, "Init() has not succeeded")
        pos = _f64(pos).reshape(-1)
        if pos.size < 3 * self.npos or f.size < 3 * self.npos:
            raise ValueError("pos and f must hold 3*npos values")
        if not (f.dtype == np.float64 and f.flags.c_contiguous):
            raise ValueError("f must be a C-contiguous float64 array")
        self._check(lib().sdt_steric_accumulate(self._h, _ptr(pos), _ptr(f)))
        return f

    def Compute(self, pos, rdi=None):
        f = np.zeros(3 * self.npos)
        return self.Accumulate(pos, rdi, f)

    def accumulate_device(self, d_pos: int, d_f: int):
        self._check(lib().sdt_steric_accumulate_device(self._h, _vp(d_pos), _vp(d_f)))

    def set_stream(self, stream_handle: int):
        self._check(lib().sdt_steric_set_stream(self._h, _vp(stream_handle)))

    def __del__(self):
        try:
            if self._h is not None:
                lib().sdt_steric_destroy(self._h)
                self._h = None
        except Exception:
            pass


class BrwnLanczos:
    """Block Lanczos sqrt(M) z in FP64 on the GPU (drop-in for BrwnLanczos)."""

    def __init__(self, dim, max_iters, max_nrhs, tol, device=0, reorth=False):
        self.dim = int(dim)
        self.max_iters = int(max_iters)
        self.max_nrhs = int(max_nrhs)
        self.tol = float(tol)
        self.device = int(device)
        self.reorth = bool(reorth)
        self._h = None
        self.last_iters = []

    def Init(self) -> bool:
        h = _vp()
        st = lib().sdt_lanczos_create(self.dim, self.max_iters, self.max_nrhs, self.tol, self.device,
                                      ctypes.byref(h))
        if st != 0:
            return False
        self._h = h
        if self.max_nrhs > self.dim // 3:
            self.max_nrhs = max(1, self.dim // 3)
        lib().sdt_lanczos_set_reorth(self._h, 1 if self.reorth else 0)
        return True

    def Compute(self, mob: MobSpme, num_rhs, ldz, z, ldy, y):
        """y[:, j] ~ sqrt(M) z[:, j]; returns the per-group iteration counts
        (-1 = not converged, which the reference only logs)."""
        if self._h is None:
            raise StokesError(-4, "Init() has not succeeded")
        z = _f64(z)
        if not isinstance(y, np.ndarray) or y.dtype != np.float64 or not y.flags["C_CONTIGUOUS"]:
            raise TypeError("y must be a C-contiguous float64 numpy array (updated in place)")
        ngroups = max(1, (int(num_rhs) + self.max_nrhs - 1) // self.max_nrhs)
        iters = (ctypes.c_int * ngroups)()
        compute = lib().sdt_lanczos_compute_ewald if isinstance(mob, MobEwald) else lib().sdt_lanczos_compute
        st = compute(self._h, mob.handle, int(num_rhs), int(ldz), _ptr(z), int(ldy), _ptr(y), iters)
        self.last_iters = list(iters)
        if st not in (0, -5):
            raise StokesError(st, lib().sdt_lanczos_last_error(self._h).decode())
        return self.last_iters

    def history(self):
        """||Y_i - Y_{i-1}||_F / ||Z||_F per iteration of the last group."""
        buf = (ctypes.c_double * 4096)()
        n = lib().sdt_lanczos_history(self._h, buf, 4096)
        return [buf[i] for i in range(min(n, 4096))]

    def products(self) -> int:
        """Block products issued by the last compute call (iterations run
        plus any issued ahead of the convergence check and discarded)."""
        out = ctypes.c_longlong(0)
        if lib().sdt_lanczos_products(self._h, ctypes.byref(out)) != 0:
            raise StokesError(-1, "sdt_lanczos_products failed")
        return int(out.value)

    def set_stream(self, stream_handle: int):
        if lib().sdt_lanczos_set_stream(self._h, _vp(stream_handle)) != 0:
            raise StokesError(-2, "sdt_lanczos_set_stream failed")

    def compute_device(self, mob: MobSpme, num_rhs, ldz, d_z: int, ldy, d_y: int):
        ngroups = max(1, (int(num_rhs) + self.max_nrhs - 1) // self.max_nrhs)
        iters = (ctypes.c_int * ngroups)()
        st = lib().sdt_lanczos_compute_device(self._h, mob.handle, int(num_rhs), int(ldz), _vp(d_z),
                                              int(ldy), _vp(d_y), iters)
        self.last_iters = list(iters)
        if st not in (0, -5):
            raise StokesError(st, lib().sdt_lanczos_last_error(self._h).decode())
        return self.last_iters

    def close(self):
        if self._h is not None:
            lib().sdt_lanczos_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BDIntegrator:
    """Device-resident BD step loop (the reference's BDSimBox::Advance,
    src/simbox/simbox_bd.cc:296-366) over a MobSpme or a MobEwald, a
    BrwnLanczos and an optional StericForce of this package (all Init()-ed,
    same device)."""

    def __init__(self, mob, brwn: BrwnLanczos, steric=None, dt=1e-3, mob_interval=16, seed=0):
        self.mob, self.brwn, self.steric = mob, brwn, steric
        self.npos = mob.npos
        h = _vp()
        create = lib().sdt_bd_create_ewald if isinstance(mob, MobEwald) else lib().sdt_bd_create
        st = create(mob.handle if isinstance(mob, MobSpme) else mob._h, brwn._h,
                    steric._h if steric is not None else None, float(dt), int(mob_interval), int(seed),
                    ctypes.byref(h))
        if st != 0:
            raise StokesError(st, "sdt_bd_create failed")
        self._h = h

    def _check(self, st):
        if st != 0:
            raise StokesError(st, lib().sdt_bd_last_error(self._h).decode())

    def set_positions(self, pos):
        pos = _f64(pos).reshape(-1)
        self._check(lib().sdt_bd_set_positions(self._h, _ptr(pos)))

    def get_positions(self):
        out = np.zeros(3 * self.npos)
        self._check(lib().sdt_bd_get_positions(self._h, _ptr(out)))
        return out

    def set_step(self, istep: int):
        self._check(lib().sdt_bd_set_step(self._h, int(istep)))

    def Advance(self, nsteps: int):
        self._check(lib().sdt_bd_advance(self._h, int(nsteps)))

    def info(self):
        istep, nc = ctypes.c_longlong(0), ctypes.c_longlong(0)
        it = (ctypes.c_int * 1)()
        self._check(lib().sdt_bd_info(self._h, ctypes.byref(istep), ctypes.byref(nc), it))
        return {"istep": istep.value, "not_converged": nc.value, "last_iters": it[0]}

    def draw_gaussian(self, step: int, nvec: int):
        n3 = 3 * self.npos
        z = np.zeros(nvec * n3)
        self._check(lib().sdt_bd_draw_gaussian(self._h, int(step), int(nvec), n3, _ptr(z)))
        return z.reshape(nvec, n3)

    def set_stream(self, stream_handle: int):
        self._check(lib().sdt_bd_set_stream(self._h, _vp(stream_handle)))

    def synchronize(self):
        self._check(lib().sdt_bd_synchronize(self._h))

    def __del__(self):
        try:
            if self._h is not None:
                lib().sdt_bd_destroy(self._h)
                self._h = None
        except Exception:
            pass


class MobSpmeBatch:
    """Many independent systems (sdt_batch_*): system s has npos[s] particles
    in a cube of edge box[s] with its own grid dim[s], xi[s] and rmax[s].
    Vectors are concatenated per system (nrhs blocks of 3*npos[s] each)."""

    def __init__(self, npos, rdi, box, dim, xi, rmax, porder=6, max_iters=100, max_nrhs=16, tol=1e-6,
                 reorth=True, lanes=8, device=0):
        self.npos = np.ascontiguousarray(npos, dtype=np.int32)
        self.nsys = len(self.npos)
        rdi = _f64(rdi).reshape(-1)
        if rdi.size != int(self.npos.sum()):
            raise ValueError("rdi must hold sum(npos) radii")
        box, xi, rmax = (np.ascontiguousarray(x, dtype=np.float64) for x in (box, xi, rmax))
        dim = np.ascontiguousarray(dim, dtype=np.int32)
        h = _vp()
        ip = ctypes.POINTER(ctypes.c_int)
        st = lib().sdt_batch_create(self.nsys, self.npos.ctypes.data_as(ip), _ptr(rdi), _ptr(box),
                                    dim.ctypes.data_as(ip), _ptr(xi), _ptr(rmax), int(porder), int(max_iters),
                                    int(max_nrhs), float(tol), 1 if reorth else 0, int(lanes), int(device),
                                    ctypes.byref(h))
        if st != 0:
            raise StokesError(st, "sdt_batch_create failed")
        self._h = h
        self.offsets = np.concatenate([[0], np.cumsum(3 * self.npos.astype(np.int64))])

    def _check(self, st, allow_nc=False):
        if st != 0 and not (allow_nc and st == -5):
            raise StokesError(st, lib().sdt_batch_last_error(self._h).decode())

    def split(self, x, nrhs=1):
        """Per-system views (nrhs, 3*npos[s]) of a concatenated vector block."""
        out = []
        for s in range(self.nsys):
            a, b = nrhs * self.offsets[s], nrhs * self.offsets[s + 1]
            out.append(x[a:b].reshape(nrhs, -1))
        return out

    def Update(self, pos):
        self._check(lib().sdt_batch_update(self._h, _ptr(_f64(pos).reshape(-1))))

    def MulVector(self, nrhs, alpha, f, beta, v):
        self._check(lib().sdt_batch_mulvec(self._h, int(nrhs), float(alpha), _ptr(f), float(beta), _ptr(v)))
        return v

    def Lanczos(self, nrhs, z, y):
        iters = (ctypes.c_int * self.nsys)()
        self._check(lib().sdt_batch_lanczos(self._h, int(nrhs), _ptr(z), _ptr(y), iters), allow_nc=True)
        return list(iters)

    def update_device(self, d_pos: int):
        self._check(lib().sdt_batch_update_device(self._h, _vp(d_pos)))

    def mulvec_device(self, nrhs, alpha, d_f: int, beta, d_v: int):
        self._check(lib().sdt_batch_mulvec_device(self._h, int(nrhs), float(alpha), _vp(d_f), float(beta),
                                                  _vp(d_v)))

    def lanczos_device(self, nrhs, d_z: int, d_y: int):
        iters = (ctypes.c_int * self.nsys)()
        self._check(lib().sdt_batch_lanczos_device(self._h, int(nrhs), _vp(d_z), _vp(d_y), iters),
                    allow_nc=True)
        return list(iters)

    def synchronize(self):
        self._check(lib().sdt_batch_synchronize(self._h))

    def set_packed(self, enable: bool):
        """Packed launches over all systems (default where supported) or
        every system's own launches spread over the lanes."""
        self._check(lib().sdt_batch_set_packed(self._h, 1 if enable else 0))

    @property
    def packed(self) -> bool:
        return lib().sdt_batch_get_packed(self._h) == 1

    def __del__(self):
        try:
            if self._h is not None:
                lib().sdt_batch_destroy(self._h)
                self._h = None
        except Exception:
            pass


class MobilityServer:
    """Served request stream (sdt_serve_*): register device-resident systems,
    submit mobility applies (kind 0) or Brownian steps (kind 1) with k RHS,
    wait for tickets.  Arrays passed to submit() are kept referenced until
    their ticket has been waited for."""

    def __init__(self, device=0, hbm_budget_bytes=64e9, lanes=4, max_npos=100000, max_iters=100,
                 max_nrhs=16, tol=1e-6):
        h = _vp()
        st = lib().sdt_serve_create(int(device), float(hbm_budget_bytes), int(lanes), int(max_npos),
                                    int(max_iters), int(max_nrhs), float(tol), ctypes.byref(h))
        if st != 0:
            raise StokesError(st, "sdt_serve_create failed")
        self._h = h
        self._keep = {}

    def _err(self):
        return lib().sdt_serve_last_error(self._h).decode()

    def register(self, npos, rdi, box, dim, xi, rmax, porder, pos) -> int:
        sid = ctypes.c_int(-1)
        st = lib().sdt_serve_register(self._h, int(npos), _ptr(_f64(rdi)), float(box), int(dim), float(xi),
                                      float(rmax), int(porder), _ptr(_f64(pos).reshape(-1)), ctypes.byref(sid))
        if st != 0:
            raise StokesError(st, self._err())
        return sid.value

    def submit(self, sys_id, kind, nrhs, x, out) -> int:
        if not (x.dtype == np.float64 and x.flags.c_contiguous and out.dtype == np.float64
                and out.flags.c_contiguous):
            raise ValueError("x and out must be C-contiguous float64 arrays")
        t = ctypes.c_longlong(-1)
        st = lib().sdt_serve_submit(self._h, int(sys_id), int(kind), int(nrhs), _ptr(x), _ptr(out),
                                    ctypes.byref(t))
        if st != 0:
            raise StokesError(st, self._err())
        self._keep[t.value] = (x, out)
        return t.value

    def wait(self, ticket, timeout_ms=600000.0):
        lat = ctypes.c_double(0.0)
        st = lib().sdt_serve_wait(self._h, int(ticket), float(timeout_ms), ctypes.byref(lat))
        if st == -4:
            raise TimeoutError(f"ticket {ticket} still pending")
        self._keep.pop(ticket, None)
        if st != 0:
            raise StokesError(st, self._err())
        return lat.value

    def stats(self):
        c, r, u = ctypes.c_longlong(0), ctypes.c_longlong(0), ctypes.c_double(0.0)
        lib().sdt_serve_stats(self._h, ctypes.byref(c), ctypes.byref(r), ctypes.byref(u))
        b, br, la = ctypes.c_longlong(0), ctypes.c_longlong(0), ctypes.c_int(0)
        lib().sdt_serve_batch_stats(self._h, ctypes.byref(b), ctypes.byref(br), ctypes.byref(la))
        return {"completed": c.value, "rejected": r.value, "used_bytes": u.value, "batches": b.value,
                "batched_requests": br.value, "batch_lanes": la.value}

    def close(self):
        if self._h is not None:
            lib().sdt_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# File I/O in the reference's formats
# ---------------------------------------------------------------------------
def read_xyz(path, model=None):
    """(pos (N, 3), rdi (N,), box (Lx, Ly, Lz), start_step, start_time) of an
    XYZ file, radii from the model file's par lines (MoleculeIO::ParseXYZ)."""
    n = ctypes.c_int(0)
    if lib().sdt_xyz_count(str(path).encode(), ctypes.byref(n)) != 0:
        raise StokesError(-1, f"cannot read {path}")
    pos = np.zeros(3 * n.value)
    rdi = np.zeros(n.value)
    box = np.zeros(3)
    step, t = ctypes.c_int(0), ctypes.c_double(0.0)
    st = lib().sdt_xyz_read(str(path).encode(), str(model).encode() if model else None, n.value, _ptr(pos),
                            _ptr(rdi), _ptr(box), ctypes.byref(step), ctypes.byref(t))
    if st != 0:
        raise StokesError(-1, f"malformed XYZ file {path}")
    return pos.reshape(-1, 3), rdi, tuple(box), step.value, t.value


def write_xyz(path, pos, box, frame=0, time=0.0, append=False):
    pos = _f64(pos).reshape(-1)
    b = _f64(np.broadcast_to(np.asarray(box, dtype=np.float64), (3,)).copy())
    if lib().sdt_xyz_write(str(path).encode(), 1 if append else 0, pos.size // 3, _ptr(b), int(frame),
                           float(time), _ptr(pos)) != 0:
        raise StokesError(-1, f"cannot write {path}")


def config_get(path, key):
    buf = ctypes.create_string_buffer(512)
    st = lib().sdt_config_get(str(path).encode(), key.encode(), buf, 512)
    if st < 0:
        raise StokesError(-1, f"cannot read {path} (or duplicate key {key})")
    return buf.value.decode() if st == 0 else None


def model_steric(path):
    r0, k0 = ctypes.c_double(0.0), ctypes.c_double(0.0)
    st = lib().sdt_model_steric(str(path).encode(), ctypes.byref(r0), ctypes.byref(k0))
    if st < 0:
        raise StokesError(-1, f"cannot read {path}")
    return (r0.value, k0.value) if st == 0 else None
