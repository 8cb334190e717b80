"""The C++ drop-in path: include/qlgpu.hpp (Model / Integrator / solution
mirror) driven by csrc/examples/ql_main.cpp, which reads the reference's
.DSSinput keys, checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from gpu_util import rel, require_gpu
from oracle import oracle as O
from ql_dns_b200.build import MAIN, build
from ql_dns_b200.initial import initial_state
from ql_dns_b200.params import mri_16x16_nz32

pytestmark = pytest.mark.gpu


def write_input(path, p, integ, tv_every):
    name = "MHD_BQlin" if p.model == 0 else "MHD_FullQlin"
    txt = f"""equations_to_use_ = {name}
nx_ = {p.nx}
ny_ = {p.ny}
nz_ = {p.NZ}
lx_ = {p.L[0]!r}
ly_ = {p.L[1]!r}
lz_ = {p.L[2]!r}
dt_ = {p.dt!r}
tv_save_ = {p.dt * tv_every!r}
nu_ = {p.nu!r}
eta_ = {p.eta!r}
viscosity_order_ = {p.viscosity_order}
q_ = {p.q!r}
omega_ = {p.omega!r}
B0z_ = {p.B0z!r}
Remap? = {p.remap}
QuasiLinear? = {p.quasilinear}
integrator_ = {integ}
full_save_ = 1.0
"""
    open(path, "w").write(txt)


@pytest.mark.parametrize("integ", [0, 1])
def test_cpp_driver_matches_oracle(tmp_path, integ):
    require_gpu()
    build()
    p = mri_16x16_nz32(integrator=integ)
    lin, mf, kx0 = initial_state(p, 9, sigma=0.1)
    inp = tmp_path / "case.DSSinput"
    write_input(inp, p, integ, 1)
    st = tmp_path / "state.bin"
    with open(st, "wb") as f:
        np.array([0.0]).tofile(f)
        lin.tofile(f)
        mf.tofile(f)
        kx0.tofile(f)
    out, dg = tmp_path / "out.bin", tmp_path / "diag.bin"
    odir = tmp_path / "sim"
    odir.mkdir()
    r = subprocess.run([MAIN, str(inp), str(st), "100", str(out), str(dg), str(odir)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(out, dtype=np.float64)
    n_lin, n_mf = lin.size * 2, mf.size * 2
    t = raw[0]
    lo = raw[1:1 + n_lin].view(np.complex128).reshape(lin.shape)
    mo = raw[1 + n_lin:1 + n_lin + n_mf].view(np.complex128).reshape(mf.shape)
    ko = raw[1 + n_lin + n_mf:]
    d = np.fromfile(dg, dtype=np.float64).reshape(-1, 15)
    t2, lo2, mo2, ko2, d2 = O.run(p, 0.0, lin, mf, kx0, 100, diag_every=1)
    assert t == t2 and np.array_equal(ko, ko2)
    assert rel(lo, lo2) < 1e-10 and rel(mo, mo2) < 1e-10
    assert d.shape == d2.shape and rel(d[:, 1:13], d2[:, 1:13]) < 1e-10
    # the reference's output files from the same run
    from ql_dns_b200 import io
    e = np.fromfile(odir / "energy.dat").reshape(-1, 4)
    assert np.array_equal(e, d[:, 1:5]) and np.array_equal(np.fromfile(odir / "time_vec.dat"), d[:, 0])
    assert np.fromfile(odir / "mean_fields.dat").size == 2 * p.nmf * p.NZ
    tl, ll, ml, kl = io.load_solution(str(odir / "FullSave.bin"), p)
    assert tl == t and np.array_equal(ll, lo.astype(np.complex64).astype(np.complex128))
    assert np.array_equal(ml, mo.astype(np.complex64).astype(np.complex128))


def test_cpp_driver_with_noise_and_cfl(tmp_path):
    # dt_ < 0 (variable dt = CFL_ / Calculate_CFL, at most |dt_|) and f_noise_ != 0
    # (DrivingNoise after every step) read from the input file, as main.cpp:112-113 and
    # RK3CN_Elin.cpp:22-27,76-80 use them
    require_gpu()
    build()
    p = mri_16x16_nz32(dt=0.02)
    lin, mf, kx0 = initial_state(p, 4, sigma=1e-3, B0=0.2)
    inp = tmp_path / "case.DSSinput"
    write_input(inp, p, 0, 5)  # tv_save_ = 5 |dt_|
    txt = open(inp).read().replace(f"dt_ = {p.dt!r}", f"dt_ = {-p.dt!r}")
    open(inp, "w").write(txt)
    with open(inp, "a") as f:
        f.write("CFL_ = 0.2\nf_noise_ = 0.05\nnoise_range_low_ = 1.0\nnoise_range_high_ = 30.0\nnoise_seed_ = 77\n")
    st = tmp_path / "state.bin"
    with open(st, "wb") as f:
        np.array([0.0]).tofile(f)
        lin.tofile(f)
        mf.tofile(f)
        kx0.tofile(f)
    out, dg = tmp_path / "out.bin", tmp_path / "diag.bin"
    r = subprocess.run([MAIN, str(inp), str(st), "40", str(out), str(dg)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(out, dtype=np.float64)
    n_lin, n_mf = lin.size * 2, mf.size * 2
    t = raw[0]
    lo = raw[1:1 + n_lin].view(np.complex128).reshape(lin.shape)
    mo = raw[1 + n_lin:1 + n_lin + n_mf].view(np.complex128).reshape(mf.shape)
    d = np.fromfile(dg, dtype=np.float64).reshape(-1, 15)
    t2, lo2, mo2, ko2, d2, dtm = O.run_forced(p, 0.0, lin, mf, kx0, 40, diag_every=5, cfl=0.2, dt_max=0.02,
                                             f_noise=0.05, k_lo=1.0, k_hi=30.0, seed=77)
    assert dtm < 0.02 and abs(t - t2) <= 1e-13 * t2
    assert rel(lo, lo2) < 1e-10 and rel(mo, mo2) < 1e-10
    assert d.shape == d2.shape and rel(d[:, 1:13], d2[:, 1:13]) < 1e-10
