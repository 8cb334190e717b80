"""Output and restart files (include/qlgpu_io.h) against independent numpy
readers of the reference's layouts: TimeVariables.cpp (.dat files) and
FullSave_Load.cpp (groups and dataset names, float32 data).  No GPU."""
import os
import struct

import numpy as np
import pytest

from ql_dns_b200 import _capi, io
from ql_dns_b200.build import build
from ql_dns_b200.initial import initial_state
from ql_dns_b200.ktables import ktables
from ql_dns_b200.params import mri_16x16_nz32


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build()
    _capi.load()


def padded_inverse_real(f, NZ):
    """fac1D * real(inverse(f)) with the fftwPlans padding (fftwPlans.cpp:29-34)."""
    nz = f.shape[-1]
    low = (nz - 1) // 2 + 1
    pad = np.zeros(NZ, dtype=complex)
    pad[:low] = f[:low]
    pad[NZ - (nz - low):] = f[low:]
    return np.fft.ifft(pad).real  # numpy's ifft is the backward sign times 1/NZ


def test_timevariables_files(tmp_path):
    p = mri_16x16_nz32(nx=8, ny=8, NZ=32)
    d = str(tmp_path) + "/"
    rng = np.random.default_rng(3)
    recs = rng.normal(size=(3, 15))
    _, mf, _ = initial_state(p, 1, sigma=0.1)
    mf2 = mf * 1.5 + 0.01j
    with io.TimeVariables(d, p) as tv:
        tv.save_mean_fields(mf)
        for r in recs:
            tv.save_data(r)
        tv.save_mean_fields(mf2)
    e = np.fromfile(d + "energy.dat").reshape(-1, 4)
    am = np.fromfile(d + "angular_momentum.dat").reshape(-1, 4)
    di = np.fromfile(d + "dissipation.dat").reshape(-1, 4)
    tv_ = np.fromfile(d + "time_vec.dat")
    rey = np.fromfile(d + "reynolds_stress.dat").reshape(-1, 5)
    mfd = np.fromfile(d + "mean_fields.dat").reshape(-1, p.nmf, p.NZ)
    assert np.array_equal(e, recs[:, 1:5]) and np.array_equal(am, recs[:, 5:9])
    assert np.array_equal(di, recs[:, 9:13]) and np.array_equal(tv_, recs[:, 0])
    assert rey.shape == (3, 5) and not rey.any()
    assert mfd.shape == (2, 2, 32)
    for k, m in enumerate([mf, mf2]):
        for i in range(p.nmf):
            assert np.allclose(mfd[k, i], padded_inverse_real(m[i], p.NZ), rtol=0, atol=1e-14 * np.abs(m).max())
    # append keeps, truncate clears
    with io.TimeVariables(d, p, append=True) as tv:
        tv.save_data(recs[0])
    assert np.fromfile(d + "time_vec.dat").size == 4
    with io.TimeVariables(d, p, append=False):
        pass
    assert os.path.getsize(d + "energy.dat") == 0


def parse_container(path):
    """Independent reader of the FullSave container layout."""
    b = open(path, "rb").read()
    assert b[:8] == b"QLFSAVE1"
    nlin, nz, nmf, nxy = struct.unpack_from("<4i", b, 8)
    o = 24
    groups = []
    while o < len(b):
        (n,) = struct.unpack_from("<I", b, o)
        name = b[o + 4:o + 4 + n].decode()
        o += 4 + n
        (t,) = struct.unpack_from("<d", b, o)
        (nds,) = struct.unpack_from("<I", b, o + 8)
        o += 12
        ds = {}
        for _ in range(nds):
            (n,) = struct.unpack_from("<I", b, o)
            dn = b[o + 4:o + 4 + n].decode()
            o += 4 + n
            typ, cnt = struct.unpack_from("<IQ", b, o)
            o += 12
            if typ == 0:
                arr = np.frombuffer(b, dtype=np.complex64, count=cnt, offset=o)
                o += 8 * cnt
            else:
                arr = np.frombuffer(b, dtype=np.float32, count=cnt, offset=o)
                o += 4 * cnt
            ds[dn] = arr
        groups.append((name, t, ds))
    return (nlin, nz, nmf, nxy), groups


@pytest.mark.parametrize("model", [0, 1])
def test_fullsave_layout_and_restart(tmp_path, model):
    p = mri_16x16_nz32(nx=8, ny=6, NZ=32, model=model)
    path = str(tmp_path / "full.bin")
    kt = ktables(p)
    lin, mf, kx0 = initial_state(p, 4, sigma=0.3)
    kx0b = kx0 - 3 * (2 * np.pi / p.L[0]) * (kt["ky"] > 0)  # a remapped state
    io.save_solution(path, p, 0.5, lin * 0.5, mf * 0.5, kx0)
    io.save_solution(path, p, 1.25, lin, mf, kx0b)
    dims, groups = parse_container(path)
    assert dims == (4, p.nz, p.nmf, p.nxy)
    assert [g[0] for g in groups] == ["/t=0.5", "/t=1.25"]
    name, t, ds = groups[1]
    assert len(ds) == p.nxy + 2
    for j in range(p.nxy):
        key = f"Ind {j}: kx {kt['kx_index'][j]} ky {kt['ky_index'][j]}"
        assert np.array_equal(ds[key], lin[j].reshape(-1).astype(np.complex64))
    assert np.array_equal(ds["Mean"], mf.reshape(-1).astype(np.complex64))
    assert np.array_equal(ds["kx"], (kx0b + p.q * 1.25 * kt["ky"]).astype(np.float32))
    assert io.saved_times(path) == [0.5, 1.25]
    t, lo, mo, ko = io.load_solution(path, p)
    assert t == 1.25
    assert np.array_equal(lo, lin.astype(np.complex64).astype(np.complex128))
    assert np.array_equal(mo, mf.astype(np.complex64).astype(np.complex128))
    kf = (kx0b + p.q * 1.25 * kt["ky"]).astype(np.float32).astype(np.float64)
    assert np.array_equal(ko, kf - p.q * 1.25 * kt["ky"])
    assert np.abs(ko - kx0b).max() < 1e-5 * np.abs(kx0b).max()


def test_fullsave_rejects_mismatch(tmp_path):
    p = mri_16x16_nz32(nx=8, ny=8, NZ=32)
    path = str(tmp_path / "full.bin")
    lin, mf, kx0 = initial_state(p, 4, sigma=0.3)
    io.save_solution(path, p, 0.1, lin, mf, kx0)
    with pytest.raises(_capi.QLGPUError) as ei:
        io.load_solution(path, p.replace(NZ=64))
    assert "do not match" in str(ei.value)
    with pytest.raises(_capi.QLGPUError):
        io.load_solution(str(tmp_path / "missing.bin"), p)


def _write_container(path, p, t, datasets):
    """A FullSave container with one group holding the given (name, type, float32 payload) datasets."""
    b = bytearray(b"QLFSAVE1")
    b += struct.pack("<4i", 4, p.nz, p.nmf, p.nxy)
    name = f"/t={t}".encode()
    b += struct.pack("<I", len(name)) + name + struct.pack("<dI", t, len(datasets))
    for dn, typ, payload in datasets:
        dn = dn.encode()
        cnt = payload.size // 2 if typ == 0 else payload.size
        b += struct.pack("<I", len(dn)) + dn + struct.pack("<IQ", typ, cnt) + payload.astype(np.float32).tobytes()
    open(path, "wb").write(bytes(b))


def test_fullsave_rejects_corrupt_and_incomplete_groups(tmp_path):
    p = mri_16x16_nz32(nx=4, ny=4, NZ=16)
    kt = ktables(p)
    lin, mf, kx0 = initial_state(p, 5, sigma=0.3)
    good = [(f"Ind {j}: kx {kt['kx_index'][j]} ky {kt['ky_index'][j]}", 0,
             lin[j].reshape(-1).view(np.float64)) for j in range(p.nxy)]
    mean = ("Mean", 0, mf.reshape(-1).view(np.float64))
    kxd = ("kx", 1, kx0 + p.q * 0.5 * kt["ky"])
    path = str(tmp_path / "ok.bin")
    _write_container(path, p, 0.5, good + [mean, kxd])
    t, lo, mo, ko = io.load_solution(path, p)
    assert t == 0.5 and np.abs(lo - lin).max() < 1e-6 * np.abs(lin).max()
    # a mode dataset missing from the group
    path = str(tmp_path / "missing_ind.bin")
    _write_container(path, p, 0.5, good[:2] + good[3:] + [mean, kxd])
    with pytest.raises(_capi.QLGPUError) as ei:
        io.load_solution(path, p)
    assert "Ind 2" in str(ei.value)
    # no mean fields
    path = str(tmp_path / "missing_mean.bin")
    _write_container(path, p, 0.5, good + [kxd])
    with pytest.raises(_capi.QLGPUError) as ei:
        io.load_solution(path, p)
    assert "Mean" in str(ei.value)
    # the last dataset's count patched to an absurd size: an error, not an allocation failure
    path = str(tmp_path / "corrupt.bin")
    _write_container(path, p, 0.5, good + [mean, kxd])
    raw = bytearray(open(path, "rb").read())
    off = raw.rfind(b"kx") + 2 + 4  # name, then the type word; the count follows
    struct.pack_into("<Q", raw, off, 1 << 61)
    open(path, "wb").write(bytes(raw))
    with pytest.raises(_capi.QLGPUError):
        io.load_solution(path, p)
