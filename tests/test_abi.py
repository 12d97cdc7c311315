"""CPU checks of the C ABI: the library loads, exports every declared symbol, and its host-only
entry points (defaults, input.inp parser, argument validation) behave without a GPU."""
import ctypes
import os
import re

import pytest

from mhit36_mixedp_b200 import _lib, api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mhit_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(mhit_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding knows all of them
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def struct_fields(src, name):
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), src, flags=re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    out = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        names = decl.split(None, 1)[1] if not decl.startswith("long long") else decl.split(None, 2)[2]
        for n in names.split(","):
            out.append(re.sub(r"\[.*\]", "", n).strip())
    return out


def test_ctypes_structs_match_header():
    src = open(HEADER).read()
    assert struct_fields(src, "mhit_params") == [f for f, _ in _lib.MhitParams._fields_]
    assert struct_fields(src, "mhit_run") == [f for f, _ in _lib.MhitRun._fields_]
    assert struct_fields(src, "mhit_diag") == [f for f, _ in _lib.MhitDiag._fields_]


def test_fortran_module_matches_header():
    f90 = open(os.path.join(ROOT, "mhit36_mixedp_b200", "fortran", "mhit_gpu.f90")).read()
    body = re.search(r"type, bind\(C\) :: mhit_params(.*?)end type", f90, flags=re.S).group(1)
    names = []
    for line in body.splitlines():
        if "::" in line:
            names += [n.strip() for n in line.split("::")[1].split(",")]
    assert names == [f for f, _ in _lib.MhitParams._fields_]
    # every C entry point used by a Fortran host is bound
    for fn in ("mhit_init", "mhit_step", "mhit_upload_fields", "mhit_download_fields", "mhit_read_input",
               "mhit_write_field", "mhit_read_field", "mhit_diagnostics", "mhit_destroy",
               "mhit_ensemble_create", "mhit_ensemble_box", "mhit_ensemble_step", "mhit_ensemble_autotune",
               "mhit_ensemble_destroy", "mhit_init_taylor_green", "mhit_init_velocity_modes", "mhit_init_drops",
               "mhit_energy_spectrum", "mhit_init_particles"):
        assert f'name="{fn}"' in f90, fn
    # the Poisson-mode constants agree with the C side
    for name, val in (("MHIT_POISSON_FP64", 0), ("MHIT_POISSON_FP32", 1), ("MHIT_POISSON_FP32_REFINED", 2)):
        assert re.search(rf"\b{name} = {val}\b", f90), name
        assert _lib.POISSON[name.split("MHIT_POISSON_")[1].lower()] == val


def test_abi_version():
    assert api.abi_version() == 1


def test_params_default_matches_reference_input():
    c = _lib.MhitParams()
    assert _lib.load().mhit_params_default(ctypes.byref(c)) == 0
    # multi/input.inp:7-16
    assert (c.dt, c.mu, c.rho, c.f1, c.f2, c.f3, c.k0) == (0.0002, 0.006, 1.0, 1.0, 1.0, 1.0, 2.0)
    assert (c.radius, c.sigma, c.epsr) == (0.5, 1.0, 1.0)
    assert c.poisson == 0 and c.laplacian == 0 and c.yz_shift == 1


INPUT_INP = """0           ! fresh start=0 restart =1
0           ! iteration to start from (fresh start 0 otherwise different)
10000           ! Final time step
100000           ! Saving frequency
0           ! inflow condition (0=Taylor green, 1=read from fields)
0           ! phase-field initial condition (0=circular drop, 1=read from fields)
0.0002      ! dt for the simulation
0.006       ! mu (viscosity)
1.000       ! density
1.0         ! A forcing parameter (ABC forcing)
1.0         ! B forcing parameter (ABC forcing)
1.0         ! C forcing parameter (ABC forcing)
2.0         ! Forced wavenumber (ABC forcing)
0.5         ! Initial drop radius for phase-field
1.0d0       ! Surface tension
1.0         ! Ratio eps/dx
10000       ! Number particles
1           ! Particle initial condition (0 from file, 1 random, 2 random in drops)
"""


def test_read_input(tmp_path):
    p = tmp_path / "input.inp"
    p.write_text(INPUT_INP.replace("1.0d0", "2.5D-1"))
    prm, run = api.read_input(str(p), nx=128)
    assert run == {"restart": 0, "tstart": 0, "tfin": 10000, "dump": 100000, "inflow": 0, "inphi": 0, "inpart": 1}
    assert prm.nx == 128 and prm.dt == 0.0002 and prm.mu == 0.006 and prm.sigma == 0.25
    assert prm.npart == 10000 and prm.k0 == 2.0


def test_read_input_errors(tmp_path):
    with pytest.raises(api.MhitIOError):
        api.read_input(str(tmp_path / "missing.inp"))
    p = tmp_path / "short.inp"
    p.write_text("\n".join(INPUT_INP.splitlines()[:10]) + "\n")
    with pytest.raises(api.MhitIOError, match="missing line 11"):
        api.read_input(str(p))
    p.write_text(INPUT_INP.replace("0.006 ", "abc "))
    with pytest.raises(api.MhitIOError, match="not a number"):
        api.read_input(str(p))


@pytest.mark.parametrize("bad", [dict(nx=100), dict(nx=2048), dict(dt=-1.0), dict(poisson="fp16"),
                                 dict(poisson="fp32_incremental"), dict(zsolve_tc=1, poisson="fp32"),
                                 dict(zsolve_tc=1, nz=512, poisson="fp64"), dict(zsolve_tc=2, nz=512, poisson="fp32")])
def test_init_rejects_bad_params(bad):
    kw = dict(nx=32)
    kw.update(bad)
    if kw.get("poisson") == "fp16":
        with pytest.raises(KeyError):
            api.Params(**kw).to_c()
        return
    with pytest.raises(api.MhitArgError):
        api.Solver(api.Params(**kw))


def test_init_without_gpu_fails_cleanly():
    """On a machine without a CUDA device mhit_init reports an error instead of crashing."""
    from tests.conftest import have_gpu
    if have_gpu():
        pytest.skip("a GPU is present")
    with pytest.raises(api.MhitError):
        api.Solver(api.Params(nx=32))


def test_entry_points_reject_a_null_context():
    """Every context entry point validates its handle before touching the device."""
    lib = _lib.load()
    buf = (ctypes.c_double * 64)()
    calls = {
        "mhit_step": (None, 1),
        "mhit_init_taylor_green": (None,),
        "mhit_init_velocity_modes": (None, 1, buf, 1.0),
        "mhit_init_drops": (None, 1, buf, 0.5),
        "mhit_init_particles": (None, 10, 1),
        "mhit_energy_spectrum": (None, buf, 8),
        "mhit_diagnostics": (None, None),
        "mhit_label_drops": (None, 0.5, 6, None, 0, None, None),
    }
    for name, args in calls.items():
        assert getattr(lib, name)(*args) == _lib.MHIT_ERR_ARG, name
