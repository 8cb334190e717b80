"""CPU oracle of the 3-D shearing-box MHD DNS (numpy, FP64).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the ql_dns_b200 package.

The reference has no 3-D model (its only transforms are the 1-D z plans of
QL_DNS/Auxiliary/fftwPlans.cpp:48-51), so this is the project's own
restatement of the full nonlinear system whose quasi-linear truncation is
MHD_FullQlin (QL_DNS/Models/MHD_FullQlin.cpp:171-456).  It is pinned by:

* the QL projection (``ql=True``): keeping only the mean x fluctuation products
  and the mean part of the fluctuation x fluctuation products reproduces the
  MHD_FullQlin restatement of oracle/ql_oracle.cpp to round-off, state and
  diagnostics, through remaps (tests/test_dns_oracle.py);
* ideal invariants of the full nonlinear terms (energy, cross helicity,
  magnetic helicity transfer), Hermitian symmetry and divergence-freeness.

Equations (shearing-wave frame, kx(t) = kx0 + q t ky as in
QL_DNS/Models/MHD_BQlin.cpp:498):
    du/dt = P[-i k.T + (2 Om u_y, (q - 2 Om) u_x, 0) + i kz B0z b] - k q ky u_x / k^2
    db/dt = i k x E + (0, -q b_x, 0) + i kz B0z u
with T_ij = u_i u_j - b_i b_j and E = u x b (products in real space, u and b
including the mean column), P = I - k k^T / k^2 (identity on z-removal at
k = 0), dissipation -nu |k|^order on u and -eta |k|^order on b (ordinary diffusion
-nu kz^2, -eta kz^2 on the kx = ky = 0 column, as MHD_FullQlin's mean fields)
handled by the integrators exactly as RK3CN_Elin / RK3CN (QL_DNS/Integrators/RK3CN_Elin.cpp:
74-188, RK3CN.cpp:77-202) with the operator at kx(t + dt_lin)
(MHD_FullQlin.cpp:371-376).  After every stage update the new state is
(i) zeroed where |kx(t')| > Mx/3 (2 pi/Lx) at the next evaluation time t'
(2/3 rule in the sheared frame; off in ql mode) and (ii) made divergence-free
at k(t') by removing k.u along (0, ky, kz) (u_x and the x vorticity are kept,
the reconstruction of MHD_FullQlin.cpp:220-242), or u_x = 0 where ky = kz = 0.
The remap is MHD_FullQlin.cpp:464-481 applied to whole columns.

Layout: lin[nxy, 6, nz] = (u_x, u_y, u_z, b_x, b_y, b_z) per (kx, ky) column
in the Kdata order of the QL models; column 0 is kx = ky = 0 (the means).
Stored values are physical Fourier amplitudes times Mx*My*NZ.
"""
from __future__ import annotations

import math

import numpy as np

A0, A1, A2 = 8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0
B1, B2 = -17.0 / 60.0, -5.0 / 12.0
P1, P2 = 8.0 / 15.0, 2.0 / 3.0


def kdata(q) -> dict:
    """Wavenumber tables of the (kx, ky) columns and of kz, restated from
    QL_DNS/Auxiliary/Kdata.cpp:24-46 (columns ordered j + (Ny/2) i: kx integers
    0 .. Nx/2-1 then -(Nx/2-1) .. -1, the Nyquist column dropped; ky integers
    0 .. Ny/2-1) and Kdata.cpp:74-78 (kz integers 0 .. (nz-1)/2 then
    -(nz-1)/2 .. -1).  The oracle keeps its own copy so that a table error in the
    package cannot hide in both the initial state and its check."""
    nxh, nyh = q.nx // 2, (q.ny // 2 * 2) // 2
    ix = np.concatenate([np.arange(nxh), np.arange(1 - nxh, 0)])
    kxi = np.repeat(ix, nyh)
    kyi = np.tile(np.arange(nyh), ix.size)
    nzl = (q.nz - 1) // 2
    kzi = np.concatenate([np.arange(nzl + 1), np.arange(-nzl, 0)])
    return {"kx": kxi * (2 * math.pi / q.L[0]), "ky": kyi * (2 * math.pi / q.L[1]), "kx_index": kxi,
            "ky_index": kyi, "kz": kzi * (2 * math.pi / q.L[2])}


class DNSOracle:
    def __init__(self, p):
        self.p = p
        q = p.ql()
        kt = kdata(q)
        self.kt = kt
        self.nxy, self.nz, self.nx, self.ny = q.nxy, q.nz, q.nx, q.ny
        self.Kyn = q.ny // 2
        self.ky = kt["ky"]
        self.kz = kt["kz"]
        self.kyi = kt["ky_index"].astype(np.int64)
        self.dkx = 2 * math.pi / p.L[0]
        kzL = 2 * math.pi / p.L[2]
        self.kzi = np.rint(self.kz / kzL).astype(np.int64)
        self.zbin = self.kzi % p.NZ
        assert kt["kx_index"][0] == 0 and kt["ky_index"][0] == 0
        self.norm = float(p.Mx * p.My * p.NZ)

    # ---- transforms -------------------------------------------------------
    def xbins(self, kx0):
        return np.rint(np.asarray(kx0) / self.dkx).astype(np.int64) % self.p.Mx

    def to_phys(self, lin, kx0):
        """Real fields [nf, Mx, My, NZ] of spectral columns lin[nxy, nf, nz]."""
        p = self.p
        nf = lin.shape[1]
        S = np.zeros((nf, p.Mx, p.My // 2 + 1, p.NZ), dtype=np.complex128)
        bx = self.xbins(kx0)
        S[:, bx[:, None], self.kyi[:, None], self.zbin[None, :]] = np.transpose(lin, (1, 0, 2))
        S = np.fft.ifft(S, axis=1)
        S = np.fft.ifft(S, axis=3)
        return np.fft.irfft(S, n=p.My, axis=2)

    def from_phys(self, f, kx0):
        """Spectral columns [nxy, nf, nz] (unnormalised forward) of real fields."""
        F = np.fft.rfft(f, axis=2)
        F = np.fft.fft(F, axis=1)
        F = np.fft.fft(F, axis=3)
        bx = self.xbins(kx0)
        return np.transpose(F[:, bx[:, None], self.kyi[:, None], self.zbin[None, :]], (1, 0, 2)).copy()

    @staticmethod
    def products(ph):
        """T_xx, T_yy, T_zz, T_xy, T_xz, T_yz (u_i u_j - b_i b_j), E = u x b."""
        ux, uy, uz, bx, by, bz = ph
        return np.stack([ux * ux - bx * bx, uy * uy - by * by, uz * uz - bz * bz,
                         ux * uy - bx * by, ux * uz - bx * bz, uy * uz - by * bz,
                         uy * bz - uz * by, uz * bx - ux * bz, ux * by - uy * bx])

    def spectral_products(self, lin, kx0, ql=False):
        Tm = self.from_phys(self.products(self.to_phys(lin, kx0)), kx0)
        if ql:
            # drop the fluctuation part of fluctuation x fluctuation products
            fl = lin.copy()
            fl[0] = 0.0
            Tf = self.from_phys(self.products(self.to_phys(fl, kx0)), kx0)
            Tm[1:] -= Tf[1:]
        return Tm

    # ---- right-hand side --------------------------------------------------
    def kvec(self, t, kx0):
        kxt = np.asarray(kx0) + self.p.q * t * self.ky
        shape = (self.nxy, self.nz)
        return (np.broadcast_to(kxt[:, None], shape), np.broadcast_to(self.ky[:, None], shape),
                np.broadcast_to(self.kz[None, :], shape))

    def keep(self, t, kx0):
        """Column mask of the 2/3 rule in x at time t."""
        if not self.p.dealias_xy:
            return np.ones(self.nxy, dtype=bool)
        kxt = np.asarray(kx0) + self.p.q * t * self.ky
        return np.abs(kxt) <= (self.p.Mx / 3.0) * self.dkx

    def rhs(self, t, lin, kx0, ql=False):
        p = self.p
        T = self.spectral_products(lin, kx0, ql)
        Kx, Ky, Kz = self.kvec(t, kx0)
        ux, uy, uz, bx, by, bz = (lin[:, c] for c in range(6))
        Txx, Tyy, Tzz, Txy, Txz, Tyz, Ex, Ey, Ez = T[:, 0], T[:, 1], T[:, 2], T[:, 3], T[:, 4], T[:, 5], \
            T[:, 6], T[:, 7], T[:, 8]
        om, q, B0z = p.omega, p.q, p.B0z
        Ax = -1j * (Kx * Txx + Ky * Txy + Kz * Txz) + 2 * om * uy + 1j * Kz * B0z * bx
        Ay = -1j * (Kx * Txy + Ky * Tyy + Kz * Tyz) + (q - 2 * om) * ux + 1j * Kz * B0z * by
        Az = -1j * (Kx * Txz + Ky * Tyz + Kz * Tzz) + 1j * Kz * B0z * bz
        K2 = Kx * Kx + Ky * Ky + Kz * Kz
        with np.errstate(divide="ignore"):
            iK2 = np.where(K2 > 0, 1.0 / np.where(K2 > 0, K2, 1.0), 0.0)
        s = (Kx * Ax + Ky * Ay + Kz * Az + q * Ky * ux) * iK2
        F = np.empty_like(lin)
        F[:, 0] = Ax - Kx * s
        F[:, 1] = Ay - Ky * s
        F[:, 2] = Az - Kz * s
        F[:, 3] = 1j * (Ky * Ez - Kz * Ey) + 1j * Kz * B0z * ux
        F[:, 4] = 1j * (Kz * Ex - Kx * Ez) - q * bx + 1j * Kz * B0z * uy
        F[:, 5] = 1j * (Kx * Ey - Ky * Ex) + 1j * Kz * B0z * uz
        if not ql:
            F[~self.keep(t, kx0)] = 0.0
        return F

    def linop(self, t, dt_lin, kx0):
        """[nxy, 6, nz] dissipation operator at kx(t + dt_lin) (MHD_FullQlin.cpp:371-376)."""
        p = self.p
        kxt = np.asarray(kx0) + p.q * t * self.ky
        kxt = kxt + p.q * dt_lin * self.ky
        kz2 = -(self.kz * self.kz)
        lapF = -np.power(np.abs((-kxt[:, None] ** 2 - self.ky[:, None] ** 2) + kz2[None, :]),
                         float(p.viscosity_order // 2))
        L = np.empty((self.nxy, 6, self.nz))
        L[:, 0:3] = (p.nu * lapF)[:, None, :]
        L[:, 3:6] = (p.eta * lapF)[:, None, :]
        # the kx = ky = 0 column (the means): ordinary diffusion at every order, as the
        # mean-field operator of MHD_FullQlin (linOpMF = coef kz2, MHD_FullQlin.cpp:449-455)
        L[0, 0:3] = p.nu * kz2
        L[0, 3:6] = p.eta * kz2
        return L

    # ---- constraints after an update ---------------------------------------
    def constrain(self, t, lin, kx0, ql=False):
        if not ql:
            lin[~self.keep(t, kx0)] = 0.0
        Kx, Ky, Kz = self.kvec(t, kx0)
        kp2 = Ky * Ky + Kz * Kz
        with np.errstate(divide="ignore"):
            ikp = np.where(kp2 > 0, 1.0 / np.where(kp2 > 0, kp2, 1.0), 0.0)
        zonal = (kp2 == 0) & (Kx != 0)
        kzero = (kp2 == 0) & (Kx == 0)
        for b in (0, 3):
            D = Kx * lin[:, b] + Ky * lin[:, b + 1] + Kz * lin[:, b + 2]
            lin[:, b + 1] -= Ky * D * ikp
            lin[:, b + 2] -= Kz * D * ikp
            lin[:, b][zonal] = 0.0
            lin[:, b + 2][kzero] = 0.0
        return lin

    # ---- integrator -------------------------------------------------------
    def step(self, t, lin, kx0, Lold=None, ql=False):
        """One RK3 step (RK3CN_Elin / RK3CN stage order) and the remap.
        Returns (t + dt, lin, kx0, Lold) -- Lold is the CN operator carried
        across stages (RK3CN.cpp:119-122)."""
        p = self.p
        dt = p.dt
        cn = p.integrator == 1
        lc = dt / 2 if cn else dt
        lin = lin.copy()
        kx0 = np.array(kx0, dtype=np.float64)
        if cn and Lold is None:
            Lold = self.linop(t, 0.0, kx0)  # linearOPs_Init(t0) (RK3CN.cpp:57)
        stages = [(t, dt * P1, lc * A0, A0 * dt, 0.0, t + dt * P1),
                  (t + dt * P1, dt * (P2 - P1), lc * (A1 + B1), A1 * dt, B1 * dt, t + dt * P2),
                  (t + dt * P2, dt * (1.0 - P2), lc * (A2 + B2), A2 * dt, B2 * dt, t + dt)]
        Fp = None
        for ts, dtl, linC, n1, n2, tn in stages:
            F = self.rhs(ts, lin, kx0, ql)
            L = self.linop(ts, dtl, kx0)
            acc = n1 * F + (n2 * Fp if Fp is not None else 0.0)
            if cn:
                lin = (acc + (1 + linC * Lold) * lin) / (1.0 - linC * L)
                Lold = L
            else:
                lin = np.exp(linC * L) * (acc + lin)
            self.constrain(tn, lin, kx0, ql)
            Fp = F
        t = t + dt
        if p.remap:
            nxm = self.nx - 1
            kxt = kx0 + p.q * t * self.ky
            r = kxt > nxm / 2.0 * self.dkx
            kx0[r] = kx0[r] - nxm * self.dkx
            lin[r] = 0.0
        return t, lin, kx0, Lold

    def run(self, t, lin, kx0, nsteps, diag_every=0, ql=False):
        diags = []
        Lold = None
        for n in range(nsteps):
            t, lin, kx0, Lold = self.step(t, lin, kx0, Lold, ql)
            if diag_every and (n + 1) % diag_every == 0:
                diags.append(self.diagnostics(t, lin, kx0))
        return t, lin, kx0, (np.array(diags) if diag_every else None)

    # ---- diagnostics ------------------------------------------------------
    def diagnostics(self, t, lin, kx0):
        """[t, energy(MU, MB, u, b)/2, AM(MU, MB, u, b), diss(MU, MB, u, b), etaK_u, etaK_b]:
        the record of MHD_FullQlin::Calc_Energy_AM_Diss (MHD_FullQlin.cpp:487-717)
        with the full 3-D fluctuations."""
        p = self.p
        Kx, Ky, Kz = self.kvec(t, kx0)
        K2 = Kx * Kx + Ky * Ky + Kz * Kz
        w = np.where(self.ky == 0.0, 1.0, 2.0)[:, None]
        fl = np.ones(self.nxy, dtype=bool)
        fl[0] = False
        divf = p.L[2] / (self.norm * self.norm)
        e2u = (np.abs(lin[:, 0]) ** 2 + np.abs(lin[:, 1]) ** 2 + np.abs(lin[:, 2]) ** 2)
        e2b = (np.abs(lin[:, 3]) ** 2 + np.abs(lin[:, 4]) ** 2 + np.abs(lin[:, 5]) ** 2)
        Eu = (w * e2u)[fl].sum() * divf
        Eb = (w * e2b)[fl].sum() * divf
        AMu = (w * np.real(lin[:, 0] * np.conj(lin[:, 1])))[fl].sum() * divf
        AMb = (w * np.real(lin[:, 3] * np.conj(lin[:, 4])))[fl].sum() * divf
        Du = p.nu * (w * K2 * e2u)[fl].sum() * divf
        Db = p.eta * (w * K2 * e2b)[fl].sum() * divf
        m = lin[0]
        kz2 = self.kz * self.kz
        eMU = (np.abs(m[0]) ** 2 + np.abs(m[1]) ** 2).sum() * divf
        eMB = (np.abs(m[3]) ** 2 + np.abs(m[4]) ** 2).sum() * divf
        aMU = np.real(m[0] * np.conj(m[1])).sum() * divf
        aMB = np.real(m[3] * np.conj(m[4])).sum() * divf
        dMU = p.nu * (kz2 * (np.abs(m[0]) ** 2 + np.abs(m[1]) ** 2)).sum() * divf
        dMB = p.eta * (kz2 * (np.abs(m[3]) ** 2 + np.abs(m[4]) ** 2)).sum() * divf
        kzmax = 2 * math.pi / p.L[2] * (p.NZ // 3)
        with np.errstate(divide="ignore", invalid="ignore"):
            eku = (p.nu ** 3 / (dMU + Du)) ** 0.25 * kzmax
            ekb = (p.eta ** 3 / (dMB + Db)) ** 0.25 * kzmax
        return np.array([t, eMU / 2, eMB / 2, Eu / 2, Eb / 2, aMU, aMB, AMu, AMb, dMU, dMB, Du, Db, eku, ekb])


# ---- conversions to and from the MHD_FullQlin layout (for the QL pin) -------
def from_ql(p, t, lin4, mf, kx0):
    """DNS columns from a FullQlin state (u, zeta, b, eta; Bx, By, Ux, Uy),
    reconstructing u_y, u_z, b_y, b_z as MHD_FullQlin.cpp:220-265 at time t."""
    q = p.ql()
    kt = kdata(q)
    kxc = 1j * (np.asarray(kx0) + q.q * t * kt["ky"])[:, None]
    kyc = 1j * kt["ky"][:, None]
    kzc = 1j * kt["kz"][None, :]
    lap2 = -(kt["ky"][:, None] ** 2) - kt["kz"][None, :] ** 2
    il2 = np.where(lap2 != 0, 1.0 / np.where(lap2 != 0, lap2, 1.0), 1.0)
    s = float(p.Mx * p.My) / float(q.nx * (q.ny // 2 * 2))
    out = np.zeros((q.nxy, 6, q.nz), dtype=np.complex128)
    for b, (f, g) in enumerate([(lin4[:, 0], lin4[:, 1]), (lin4[:, 2], lin4[:, 3])]):
        out[:, 3 * b] = f * s
        out[:, 3 * b + 1] = ((-kyc * kxc) * f + kzc * g) * il2 * s
        out[:, 3 * b + 2] = (-kxc * kzc * f - kyc * g) * il2 * s
    out[0] = 0.0
    sm = float(p.Mx * p.My)
    out[0, 0], out[0, 1], out[0, 3], out[0, 4] = mf[2] * sm, mf[3] * sm, mf[0] * sm, mf[1] * sm
    return out


def to_ql(p, t, lin6, kx0):
    """(lin4, mf) of the FullQlin layout from DNS columns at time t."""
    q = p.ql()
    kt = kdata(q)
    kyc = 1j * kt["ky"][:, None]
    kzc = 1j * kt["kz"][None, :]
    s = float(q.nx * (q.ny // 2 * 2)) / float(p.Mx * p.My)
    lin4 = np.zeros((q.nxy, 4, q.nz), dtype=np.complex128)
    lin4[:, 0] = lin6[:, 0] * s
    lin4[:, 1] = (kzc * lin6[:, 1] - kyc * lin6[:, 2]) * s
    lin4[:, 2] = lin6[:, 3] * s
    lin4[:, 3] = (kzc * lin6[:, 4] - kyc * lin6[:, 5]) * s
    lin4[0] = 0.0
    sm = 1.0 / float(p.Mx * p.My)
    mf = np.stack([lin6[0, 3], lin6[0, 4], lin6[0, 0], lin6[0, 1]]) * sm
    return lin4, mf
