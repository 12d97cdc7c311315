"""ctypes wrapper of oracle/liboracle.so (TEST INFRASTRUCTURE ONLY: checker and CPU baseline)."""
import ctypes
import os

import numpy as np

from . import build_oracle

_c = ctypes


class OrcParams(_c.Structure):
    _fields_ = [("nx", _c.c_int), ("ny", _c.c_int), ("nz", _c.c_int)] + \
               [(f, _c.c_double) for f in ("dt", "mu", "rho", "f1", "f2", "f3", "k0", "radius", "sigma", "epsr")] + \
               [(f, _c.c_int) for f in ("phiflag", "partflag", "poisson", "laplacian", "yz_shift", "interp", "acdi_clamp")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.build()
        L = _c.CDLL(path)
        vp, dp = _c.c_void_p, _c.POINTER(_c.c_double)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [_c.POINTER(OrcParams)]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_fields.argtypes = [vp, dp, dp, dp, dp]
        L.orc_set_particles.argtypes = [vp, dp, _c.c_int]
        L.orc_get_fields.argtypes = [vp, dp, dp, dp, dp, dp]
        L.orc_get_particles.argtypes = [vp, dp]
        L.orc_step.argtypes = [vp, _c.c_int]
        L.orc_gumax.restype = _c.c_double
        L.orc_gumax.argtypes = [vp]
        L.orc_threads.restype = _c.c_int
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_c.POINTER(_c.c_double))


class COracle:
    def __init__(self, nx, poisson="fp64", laplacian="exact", interp="linear1d", yz_shift=1, **kw):
        p = OrcParams()
        p.nx = p.ny = p.nz = nx
        for f in ("dt", "mu", "rho", "f1", "f2", "f3", "k0", "radius", "sigma", "epsr"):
            setattr(p, f, float(kw.get(f, 0.0)))
        p.phiflag = int(kw.get("phiflag", 0))
        p.partflag = int(kw.get("partflag", 0))
        p.poisson = {"fp64": 0, "fp32": 1}[poisson]
        p.laplacian = {"exact": 0, "modified": 1}[laplacian]
        p.interp = {"linear1d": 0, "trilinear": 1}[interp]
        p.yz_shift = yz_shift
        p.acdi_clamp = int(kw.get("acdi_clamp", 0))
        self.n = nx
        self.phiflag = p.phiflag
        self.h = lib().orc_create(_c.byref(p))
        self.np = 0

    def set_fields(self, u, v, w, phi=None):
        a = [np.ascontiguousarray(x, dtype=np.float64) if x is not None else None for x in (u, v, w, phi)]
        lib().orc_set_fields(self.h, *[_p(x) for x in a])

    def set_particles(self, part):
        part = np.asfortranarray(part, dtype=np.float64)
        self.np = part.shape[0]
        lib().orc_set_particles(self.h, _p(part), self.np)

    def step(self, n=1):
        lib().orc_step(self.h, int(n))

    def fields(self):
        shp = (self.n,) * 3
        out = {f: np.empty(shp) for f in ("u", "v", "w", "p")}
        phi = np.empty(shp) if self.phiflag else None
        lib().orc_get_fields(self.h, _p(out["u"]), _p(out["v"]), _p(out["w"]), _p(out["p"]), _p(phi))
        if phi is not None:
            out["phi"] = phi
        return out

    def particles(self):
        out = np.empty((self.np, 12), order="F")
        lib().orc_get_particles(self.h, _p(out))
        return out

    @property
    def gumax(self):
        return lib().orc_gumax(self.h)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def threads():
    return lib().orc_threads()
