"""Python host side of the MHIT36 B200 timestep library.

Mirrors the reference's driver (``program main``, multi/main.f90) on one GPU: the parameters
are the ``input.inp`` values read by ``readinput`` (multi/readinput.f90:14-35), the state is
the module arrays of multi/module.f90:51-71 (x-fastest, no halo), field numbers follow
``writefield``/``readfield`` (1 u, 2 v, 3 w, 4 p, 5 phi; multi/readwrite.f90:21-25), and a
step is one pass of ``do t=tstart,tfin`` (multi/main.f90:456-1007).  Every call goes through
the C ABI of ``libmhit_b200.so``; errors come back as ``MhitError`` subclasses carrying the
library's status code (the reference ``stop``s on CFL > 7, multi/main.f90:1006 -- here that is
``MhitCFLError``).
"""
from __future__ import annotations

import ctypes
import math
import dataclasses

import numpy as np

from . import _lib
from ._lib import MhitDiag, MhitDrop, MhitParams, MhitRun

FIELD_U, FIELD_V, FIELD_W, FIELD_P, FIELD_PHI = 1, 2, 3, 4, 5


class MhitError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class MhitArgError(MhitError):
    pass


class MhitCudaError(MhitError):
    pass


class MhitNaNError(MhitError):
    pass


class MhitCFLError(MhitError):
    pass


class MhitIOError(MhitError):
    pass


class MhitStateError(MhitError):
    pass


class MhitTimeoutError(MhitError):
    pass


_ERRS = {
    _lib.MHIT_ERR_ARG: MhitArgError,
    _lib.MHIT_ERR_CUDA: MhitCudaError,
    _lib.MHIT_ERR_NAN: MhitNaNError,
    _lib.MHIT_ERR_CFL: MhitCFLError,
    _lib.MHIT_ERR_IO: MhitIOError,
    _lib.MHIT_ERR_STATE: MhitStateError,
    _lib.MHIT_ERR_TIMEOUT: MhitTimeoutError,
}


def _check(rc: int):
    if rc != 0:
        msg = _lib.load().mhit_last_error()
        msg = msg.decode() if msg else ""
        raise _ERRS.get(rc, MhitError)(rc, msg)


def _dptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@dataclasses.dataclass
class Params:
    """Step parameters: ``input.inp`` lines 7-17 plus grid size and switches."""
    nx: int = 64
    ny: int | None = None
    nz: int | None = None
    dt: float = 0.0002
    mu: float = 0.006
    rho: float = 1.0
    f1: float = 1.0
    f2: float = 1.0
    f3: float = 1.0
    k0: float = 2.0
    radius: float = 0.5
    sigma: float = 1.0
    epsr: float = 1.0
    phiflag: int = 0
    partflag: int = 0
    npart: int = 0
    poisson: str = "fp64"
    laplacian: str = "exact"
    interp: str = "linear1d"
    yz_shift: int = 1
    use_graph: bool = True
    acdi_clamp: int = 0
    device: int = 0
    zsolve_tc: int = 0

    def __post_init__(self):
        self.ny = self.ny or self.nx
        self.nz = self.nz or self.nx

    def to_c(self) -> MhitParams:
        c = MhitParams()
        _check(_lib.load().mhit_params_default(ctypes.byref(c)))
        for f in ("nx", "ny", "nz", "phiflag", "partflag", "npart", "yz_shift", "device", "acdi_clamp", "zsolve_tc"):
            setattr(c, f, int(getattr(self, f)))
        for f in ("dt", "mu", "rho", "f1", "f2", "f3", "k0", "radius", "sigma", "epsr"):
            setattr(c, f, float(getattr(self, f)))
        c.poisson = _lib.POISSON[self.poisson]
        c.laplacian = _lib.LAPLACIAN[self.laplacian]
        c.interp = _lib.INTERP[self.interp]
        c.use_graph = int(bool(self.use_graph))
        return c

    @property
    def shape(self):
        """numpy shape of a field: (nz, ny, nx) C order == Fortran (nx, ny, nz)."""
        return (self.nz, self.ny, self.nx)


def read_input(path: str, **overrides):
    """Parse an ``input.inp`` (multi/readinput.f90:14-35) through the library.

    Returns ``(Params, run)`` where run holds restart/tstart/tfin/dump/inflow/inphi/inpart.
    Grid size and switches come from ``overrides`` (they are compile-time in the reference).
    """
    p = Params(**overrides)
    c = p.to_c()
    r = MhitRun()
    _check(_lib.load().mhit_read_input(path.encode(), ctypes.byref(c), ctypes.byref(r)))
    for f in ("dt", "mu", "rho", "f1", "f2", "f3", "k0", "radius", "sigma", "epsr"):
        setattr(p, f, getattr(c, f))
    p.npart = c.npart
    run = {f: getattr(r, f) for f, _ in MhitRun._fields_}
    return p, run


class Solver:
    """One box on one GPU: ``init`` -> ``upload`` -> ``step`` ... -> ``download``."""

    def __init__(self, params: Params, _borrowed_ctx=None):
        self.params = params
        self._lib = _lib.load()
        self._owned = _borrowed_ctx is None
        if self._owned:
            self._ctx = ctypes.c_void_p()
            self._cp = params.to_c()
            _check(self._lib.mhit_init(ctypes.byref(self._cp), ctypes.byref(self._ctx)))
        else:
            self._ctx = _borrowed_ctx

    # -------------------------------------------------------------- lifecycle
    def close(self):
        if self._ctx and self._owned:
            self._lib.mhit_destroy(self._ctx)
        self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _field(self, a, name):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.params.shape:
            raise MhitArgError(_lib.MHIT_ERR_ARG, f"{name} has shape {a.shape}, expected {self.params.shape}")
        return a

    # -------------------------------------------------------------- state
    def upload(self, u, v, w, phi=None):
        """Set u, v, w (and phi): the fresh-start block of multi/main.f90:322-415."""
        u, v, w = self._field(u, "u"), self._field(v, "v"), self._field(w, "w")
        if phi is not None:
            phi = self._field(phi, "phi")
        _check(self._lib.mhit_upload_fields(self._ctx, _dptr(u), _dptr(v), _dptr(w), _dptr(phi)))

    # ------------------------------------------------ initial conditions built on the device
    def init_taylor_green(self):
        """Taylor-Green velocity of multi/main.f90:324-337, synthesised on the device."""
        _check(self._lib.mhit_init_taylor_green(self._ctx))

    def init_velocity_modes(self, modes, rms: float = 1.0):
        """u, v, w = Re sum_k c_k exp(i k.x) over the (2 kmax + 1)^3 integer wavenumbers of
        ``modes`` (complex, shape (3, K, K, K) ordered [component][kz][ky][kx], k from -kmax),
        each component at its face position and scaled to ``rms``; synthesised on the device."""
        m = np.asarray(modes, dtype=np.complex128)
        if m.ndim != 4 or m.shape[0] != 3 or not (m.shape[1] == m.shape[2] == m.shape[3]) or m.shape[1] % 2 == 0:
            raise MhitArgError(_lib.MHIT_ERR_ARG, "modes must be complex (3, K, K, K) with K odd")
        kmax = (m.shape[1] - 1) // 2
        flat = np.ascontiguousarray(m).view(np.float64).ravel()
        _check(self._lib.mhit_init_velocity_modes(self._ctx, kmax, _dptr(flat), float(rms)))

    def init_solenoidal(self, seed: int, kmax: int = 4, rms: float = 1.0):
        """The seeded random solenoidal velocity of ``synth.solenoidal_velocity`` (same seed, same
        amplitudes), synthesised on the device instead of the host."""
        from . import synth
        p = self.params
        self.init_velocity_modes(synth.solenoidal_modes(seed, kmax, (1.0, p.nx / p.ny, p.nx / p.nz)), rms)

    def init_drops(self, centres, radius: float):
        """phi of drops of radius ``radius`` at ``centres`` ((n, 3) x, y, z): the nearest centre by
        minimum image, eps = epsr dx (``synth.drops_phi`` / multi/main.f90:370-382), on the device."""
        c = np.ascontiguousarray(np.asarray(centres, dtype=np.float64).reshape(-1, 3))
        _check(self._lib.mhit_init_drops(self._ctx, c.shape[0], _dptr(c), float(radius)))

    def init_particles(self, npart: int, seed: int):
        """Tracer table built on the device: tags 1..npart, seeded uniform positions
        (``synth.seeded_particles`` restates the generator), zero velocities and histories."""
        _check(self._lib.mhit_init_particles(self._ctx, int(npart), int(seed) & 0xFFFFFFFFFFFFFFFF))
        self._np = int(npart)

    def upload_particles(self, part):
        """Tracer table (npart, 12): tag, x, y, z, u, v, w, phi, u1, v1, w1, phi1."""
        part = np.asfortranarray(part, dtype=np.float64)
        if part.ndim != 2 or part.shape[1] != 12:
            raise MhitArgError(_lib.MHIT_ERR_ARG, "particle table must be (npart, 12)")
        self._np = part.shape[0]
        _check(self._lib.mhit_upload_particles(self._ctx, _dptr(part), part.shape[0]))

    def download_particles(self):
        n = getattr(self, "_np", 0)
        out = np.zeros((n, 12), dtype=np.float64, order="F")
        _check(self._lib.mhit_download_particles(self._ctx, _dptr(out), n))
        return out

    def step(self, nsteps: int = 1):
        """Advance nsteps (Euler on the first step after upload, then AB2)."""
        _check(self._lib.mhit_step(self._ctx, int(nsteps)))

    def download(self, fields=("u", "v", "w", "p", "phi")):
        shp = self.params.shape
        out = {}
        ptrs = []
        for f in ("u", "v", "w", "p", "phi"):
            if f in fields and (f != "phi" or self.params.phiflag):
                out[f] = np.empty(shp, dtype=np.float64)
                ptrs.append(_dptr(out[f]))
            else:
                ptrs.append(None)
        _check(self._lib.mhit_download_fields(self._ctx, *ptrs))
        return out

    def diagnostics(self) -> dict:
        d = MhitDiag()
        _check(self._lib.mhit_diagnostics(self._ctx, ctypes.byref(d)))
        return {
            "nstep": d.nstep, "gumax": d.gumax, "cfl": d.cfl, "mean": tuple(d.mean),
            "maxdiv": d.maxdiv, "ke": d.ke, "dissipation": d.dissipation, "flags": d.flags,
        }

    def energy_spectrum(self, nbins: int | None = None) -> np.ndarray:
        """E(k), k = 0..nbins-1: shell sums of 1/2 |u_k|^2 over the FP64 FFT of the velocity
        (mean removed, normalised by nx ny nz; sum E = KE).  Default: every shell of the box."""
        if nbins is None:
            nx, ny, nz = self.params.nx, self.params.ny, self.params.nz
            nbins = int(math.ceil(math.sqrt(3.0) * max(nx, ny, nz) / 2)) + 2
        out = np.zeros(int(nbins), dtype=np.float64)
        _check(self._lib.mhit_energy_spectrum(self._ctx, _dptr(out), int(nbins)))
        return out

    # -------------------------------------------------------------- field files
    def writefield(self, outdir: str, t: int, fieldn: int):
        """``writefield(t, fieldn)``: <outdir>/{u,v,w,p,phi}_%08d.dat (multi/readwrite.f90:1-96)."""
        _check(self._lib.mhit_write_field(self._ctx, outdir.encode(), int(t), int(fieldn)))

    def readfield(self, path: str, fieldn: int):
        """``readfield(fieldn)`` / ``readfield_restart`` (multi/readwrite.f90:107-318)."""
        _check(self._lib.mhit_read_field(self._ctx, path.encode(), int(fieldn)))

    def write_checkpoint(self, path: str):
        """Everything the next step reads (fields, AB2 history, device scalars, step count,
        tracers): a run resumed with ``read_checkpoint`` continues bit for bit."""
        _check(self._lib.mhit_write_checkpoint(self._ctx, path.encode()))

    def read_checkpoint(self, path: str):
        """Restore a ``write_checkpoint`` file into a context of the same size and mode."""
        _check(self._lib.mhit_read_checkpoint(self._ctx, path.encode()))
        if self.params.partflag:
            import struct
            with open(path, "rb") as f:
                hdr = f.read(48)
            self._np = struct.unpack_from("<i", hdr, 8 + 6 * 4)[0]

    # -------------------------------------------------------------- droplet labelling
    def label_drops(self, thresh: float = 0.5, connectivity: int = 6, labels: bool = False, capacity: int = 4096):
        """Connected components of phi >= thresh with periodic boundaries and their statistics
        (post/unionfind_periodic/main.f90).  Returns a dict of arrays ordered by each drop's
        smallest cell index: cells, volume, x, y, z (circular-mean centre), u, v, w (mean
        velocity); with labels=True also the (nz, ny, nx) int32 label field (0 background)."""
        cap = max(int(capacity), 1)
        while True:
            arr = (MhitDrop * cap)()
            nd = ctypes.c_int()
            lab = np.empty(self.params.shape, dtype=np.int32) if labels else None
            lp = lab.ctypes.data_as(ctypes.c_void_p) if labels else None
            _check(self._lib.mhit_label_drops(self._ctx, float(thresh), int(connectivity), arr, cap,
                                              ctypes.byref(nd), lp))
            if nd.value <= cap:
                break
            cap = nd.value
        n = nd.value
        out = {f: np.array([getattr(arr[i], f) for i in range(n)], dtype=np.int64 if f == "cells" else np.float64)
               for f, _ in MhitDrop._fields_}
        if labels:
            out["labels"] = lab
        return out

    # -------------------------------------------------------------- measurement
    def time_steps(self, nsteps: int) -> float:
        ms = ctypes.c_double()
        _check(self._lib.mhit_time_steps(self._ctx, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def kernels_per_step(self) -> int:
        """Kernels one step after the first launches (nodes of the captured step graph)."""
        n = ctypes.c_int()
        _check(self._lib.mhit_kernels_per_step(self._ctx, ctypes.byref(n)))
        return n.value

    # -------------------------------------------------------------- test hooks
    def run_stage(self, stage: str):
        """Run one stage of the step being built (see mhit_debug_run_stage)."""
        _check(self._lib.mhit_debug_run_stage(self._ctx, _lib.STAGES.index(stage)))

    def commit_step(self):
        _check(self._lib.mhit_debug_commit_step(self._ctx))

    def buffer(self, name: str) -> np.ndarray:
        """An internal device buffer widened to float64 (fields in (nz, ny, nx) shape)."""
        which = _lib.BUFFERS.index(name)
        n = self._lib.mhit_debug_buffer_len(self._ctx, which)
        out = np.empty(int(n), dtype=np.float64)
        _check(self._lib.mhit_debug_get_buffer(self._ctx, which, _dptr(out)))
        if name == "spec":
            p = self.params
            pitch = n // (2 * p.ny * p.nz)
            c = out.reshape(p.nz, p.ny, pitch, 2)
            return (c[..., 0] + 1j * c[..., 1])[:, :, : p.nx // 2 + 1]
        return out.reshape(self.params.shape)

    def profile_step(self) -> dict:
        cap = 16
        ms = (ctypes.c_double * cap)()
        names = (ctypes.c_char_p * cap)()
        n = ctypes.c_int(cap)
        _check(self._lib.mhit_profile_step(self._ctx, ms, names, ctypes.byref(n)))
        return {names[i].decode(): ms[i] for i in range(n.value) if ms[i] >= 0}


class Ensemble:
    """Independent boxes of uneven sizes advanced together, one CUDA-graph launch per step.

    ``boxes[b]`` is a ``Solver`` view of box b (upload, download, diagnostics, field files);
    ``step`` advances all boxes.  ``autotune`` picks the kernels' z-chunks per box size and the
    number of concurrent streams; it zeroes the boxes, so call it before uploading.
    """

    def __init__(self, params_list):
        self._lib = _lib.load()
        self.params = list(params_list)
        arr = (MhitParams * len(self.params))(*[p.to_c() for p in self.params])
        self._e = ctypes.c_void_p()
        _check(self._lib.mhit_ensemble_create(arr, len(self.params), ctypes.byref(self._e)))
        self.boxes = []
        for b, p in enumerate(self.params):
            c = ctypes.c_void_p()
            _check(self._lib.mhit_ensemble_box(self._e, b, ctypes.byref(c)))
            self.boxes.append(Solver(p, _borrowed_ctx=c))

    def close(self):
        if self._e:
            for s in self.boxes:
                s.close()
            self._lib.mhit_ensemble_destroy(self._e)
            self._e = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, nsteps: int = 1):
        _check(self._lib.mhit_ensemble_step(self._e, int(nsteps)))

    def time_steps(self, nsteps: int) -> float:
        ms = ctypes.c_double()
        _check(self._lib.mhit_ensemble_time_steps(self._e, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def autotune(self, trials: int = 2) -> dict:
        n = ctypes.c_int()
        _check(self._lib.mhit_ensemble_autotune(self._e, int(trials), ctypes.byref(n)))
        return self.tuning()

    def tuning(self) -> dict:
        nb = len(self.params)
        lanes = ctypes.c_int()
        zp = (ctypes.c_int * nb)()
        zm = (ctypes.c_int * nb)()
        _check(self._lib.mhit_ensemble_tuning(self._e, ctypes.byref(lanes), zp, zm))
        on = ctypes.c_int()
        _check(self._lib.mhit_ensemble_batched(self._e, ctypes.byref(on)))
        return {"lanes": lanes.value, "zchunk_phase": list(zp), "zchunk_mom": list(zm), "batched": bool(on.value)}

    def set_batched(self, on: bool):
        """Batched schedule (phase and momentum of all boxes as one persistent launch each) or
        per-box lanes."""
        _check(self._lib.mhit_ensemble_set_batched(self._e, int(bool(on))))


def abi_version() -> int:
    return _lib.load().mhit_abi_version()
