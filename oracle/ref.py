"""Test infrastructure only (oracle): ctypes access to the reference's own CPU
path, built from its unmodified sources by ``oracle/Makefile`` into
``oracle/_ref/libstokesdt_ref.so``.

Only ``tests/``, ``__graft_entry__.smoke`` and ``bench.py``'s CPU baseline /
reference arm may use this module, and only as the checker or the timed CPU
baseline -- never as the product path.

Wrapped reference classes (paths relative to the reference project):
  MobSpme      src/mob/mob_spme.cc:19-263
  MobEwald     src/mob/mob_ewald.cc:21-165  (dense Ewald RPY matrix, default
               xi = 10^(1/6) sqrt(pi) / L when none is given, :50-52)
  BrwnLanczos  src/brwn/brwn_lanczos.cc:16-304
"""
from __future__ import annotations

import ctypes
import os
import re
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libstokesdt_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"reference oracle not built: {LIB_PATH} (run make -C oracle)")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.sdtref_spme_create.restype = vp
        L.sdtref_spme_create.argtypes = [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.sdtref_ewald_create.restype = vp
        L.sdtref_ewald_create.argtypes = [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double]
        L.sdtref_mob_update.argtypes = [vp, _dp, _dp]
        L.sdtref_mob_mulvec.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_int, _dp, ctypes.c_double, ctypes.c_int, _dp]
        L.sdtref_mob_dim.argtypes = [vp]
        L.sdtref_mob_dim.restype = ctypes.c_int
        L.sdtref_mob_destroy.argtypes = [vp]
        L.sdtref_ewald_getmatrix.argtypes = [vp, ctypes.c_int, _dp]
        L.sdtref_lanczos_create.restype = vp
        L.sdtref_lanczos_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_double]
        L.sdtref_lanczos_compute.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, _dp,
                                             ctypes.c_int, _dp]
        L.sdtref_lanczos_destroy.argtypes = [vp]
        L.sdtref_steric_create.restype = vp
        L.sdtref_steric_create.argtypes = [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double]
        L.sdtref_steric_accumulate.argtypes = [vp, _dp, _dp, _dp]
        L.sdtref_steric_destroy.argtypes = [vp]
        L.sdtref_set_log.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.sdtref_set_log.restype = ctypes.c_int
        L.sdtref_close_log.argtypes = []
        L.sdt_shim_fft_seconds.restype = ctypes.c_double
        L.sdt_shim_fft_seconds.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def pad_len(n: int) -> int:
    """PadLen(n, sizeof(double)) of src/util/common.h:61-65 (multiple of 8)."""
    return (n + 7) // 8 * 8


def shim_fft_seconds(reset: bool = False):
    """(seconds, calls) spent in the DFTI stand-in's compute calls
    (oracle/shim/dfti_fft.cc) since load or the last reset."""
    calls = ctypes.c_longlong(0)
    t = lib().sdt_shim_fft_seconds(1 if reset else 0, ctypes.byref(calls))
    return float(t), int(calls.value)


class RefMob:
    """MobSpme / MobEwald from the reference, FP64, host arrays.

    Vectors are column blocks: RHS j starts at ``j * ld`` (src/mob/mob_base.h:44-66).
    """

    def __init__(self, handle, npos: int, kind: str):
        if not handle:
            raise RuntimeError(f"reference {kind} Init() failed")
        self.h = handle
        self.npos = npos
        self.kind = kind

    @classmethod
    def spme(cls, rdi, box, xi, rmax, dim, porder):
        rdi = np.ascontiguousarray(rdi, dtype=np.float64)
        h = lib().sdtref_spme_create(len(rdi), _ptr(rdi), box, xi, rmax, dim, porder)
        return cls(h, len(rdi), "MobSpme")

    @classmethod
    def ewald(cls, rdi, box, tol=1e-12, xi=0.0):
        rdi = np.ascontiguousarray(rdi, dtype=np.float64)
        h = lib().sdtref_ewald_create(len(rdi), _ptr(rdi), box, tol, xi)
        return cls(h, len(rdi), "MobEwald")

    def update(self, pos, rdi):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        rdi = np.ascontiguousarray(rdi, dtype=np.float64)
        lib().sdtref_mob_update(self.h, _ptr(pos), _ptr(rdi))

    @property
    def dim(self) -> int:
        return lib().sdtref_mob_dim(self.h)

    def mulvec(self, f, alpha=1.0, beta=0.0, v=None, mode=0):
        """v := alpha*M*f + beta*v; f, v are (nrhs, ld) C arrays (ld >= 3N)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        if f.ndim == 1:
            f = f[None, :]
        nrhs, ld = f.shape
        out = np.zeros_like(f) if v is None else np.ascontiguousarray(v, dtype=np.float64).copy()
        if out.ndim == 1:
            out = out[None, :]
        lib().sdtref_mob_mulvec(self.h, mode, nrhs, alpha, ld, _ptr(f), beta, out.shape[1],
                                _ptr(out))
        return out

    def matrix(self) -> np.ndarray:
        n = self.dim
        m = np.zeros((n, n), dtype=np.float64)
        lib().sdtref_ewald_getmatrix(self.h, n, _ptr(m))
        return m

    def close(self):
        if self.h:
            lib().sdtref_mob_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefLanczos:
    """BrwnLanczos (src/brwn/brwn_lanczos.cc).  ``compute`` returns Y and the
    iteration counts the reference logs (-1 = not converged)."""

    def __init__(self, dim, max_iters=100, max_nrhs=16, tol=1e-6):
        self.h = lib().sdtref_lanczos_create(dim, max_iters, max_nrhs, tol)
        if not self.h:
            raise RuntimeError("reference BrwnLanczos Init() failed")
        self.dim = dim

    def compute(self, mob: RefMob, z: np.ndarray):
        z = np.ascontiguousarray(z, dtype=np.float64)
        if z.ndim == 1:
            z = z[None, :]
        nrhs, ld = z.shape
        # BlockLanczos writes Y with ld = PadLen(dim) (brwn_lanczos.cc:184-186)
        assert ld == pad_len(self.dim), "reference requires ldy == PadLen(3N)"
        y = np.zeros_like(z)
        fd, path = tempfile.mkstemp(prefix="sdtref_", suffix=".log")
        os.close(fd)
        try:
            lib().sdtref_set_log(path.encode(), 3)
            lib().sdtref_lanczos_compute(self.h, mob.h, nrhs, ld, _ptr(z), ld, _ptr(y))
            lib().sdtref_close_log()
            with open(path) as fh:
                text = fh.read()
        finally:
            os.unlink(path)
        iters = [int(m) for m in re.findall(r"converged in (\d+) steps", text)]
        iters += [-1] * len(re.findall(r"NOT converged", text))
        return y, iters

    def close(self):
        if self.h:
            lib().sdtref_lanczos_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def parse_xyz(path: str, radii: dict | None = None):
    """XYZ reader with the semantics of MoleculeIO::ParseXYZ
    (src/util/molecule_io.cc:141-231): line 1 = N, line 2 = "step time Lx Ly Lz",
    then "type x y z"; a type missing from ``radii`` gets radius 1.0."""
    radii = radii or {}
    with open(path) as fh:
        lines = fh.read().splitlines()
    n = int(lines[0].split()[0])
    hdr = lines[1].split()
    box = float(hdr[2])
    pos, rdi = [], []
    for ln in lines[2:]:
        t = ln.split()
        if len(t) < 4:
            continue
        pos.append([float(t[1]), float(t[2]), float(t[3])])
        rdi.append(float(radii.get(t[0], 1.0)))
    assert len(pos) == n
    return np.array(pos, dtype=np.float64), np.array(rdi, dtype=np.float64), box


def parse_mod(path: str) -> dict:
    """``par name radius charge`` lines of a .mod file (src/util/molecule_io.cc:145-158)."""
    out = {}
    with open(path) as fh:
        for ln in fh:
            t = ln.split()
            if len(t) >= 3 and t[0] == "par":
                out[t[1]] = float(t[2])
    return out


class RefSteric:
    """StericForce over PairListS (src/force/force_steric.cc:14-112,
    src/pairlist/pair_s.cc:99-186): ``accumulate`` returns f + steric(pos)."""

    def __init__(self, rdi, box, r0, k0):
        rdi = np.ascontiguousarray(rdi, dtype=np.float64)
        self.rdi = rdi
        self.h = lib().sdtref_steric_create(len(rdi), _ptr(rdi), box, r0, k0)
        if not self.h:
            raise RuntimeError("reference StericForce Init() failed")

    def accumulate(self, pos, f):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        out = np.ascontiguousarray(f, dtype=np.float64).reshape(-1).copy()
        lib().sdtref_steric_accumulate(self.h, _ptr(pos), _ptr(self.rdi), _ptr(out))
        return out

    def close(self):
        if self.h:
            lib().sdtref_steric_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
