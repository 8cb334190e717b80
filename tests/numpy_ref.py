"""Independent numpy restatement of one quasi-linear rhs and RK3 step.

Test infrastructure: a second, vectorised implementation written directly from
the reference equations (QL_DNS/Models/MHD_BQlin.cpp:117-284,
QL_DNS/Models/MHD_FullQlin.cpp:171-427, QL_DNS/Integrators/RK3CN_Elin.cpp:74-188,
QL_DNS/Integrators/RK3CN.cpp:77-202) with numpy.fft for the z transforms.
It pins the C++ oracle's transform, dealiasing and sign conventions; it is
slow-ish and only used at small sizes.
"""
from __future__ import annotations

import numpy as np

from ql_dns_b200.initial import dealias_indices
from ql_dns_b200.ktables import ktables


class NumpyQL:
    def __init__(self, p):
        self.p = p
        kt = ktables(p)
        self.kx0 = kt["kx"]
        self.ky = kt["ky"]
        self.kxi = kt["kx_index"]
        self.kyi = kt["ky_index"]
        self.kz = kt["kz"]
        self.NZ = p.NZ
        self.nz = p.nz
        self.idx = dealias_indices(p.NZ, p.nz)
        self.kz2 = -self.kz ** 2
        Ny = p.ny // 2 * 2
        self.rs_fac = 1.0 / (Ny * p.nx) ** 2
        # lap2 per ky with the ky=0, kz=0 fix (Kdata.cpp:100-119)
        self.lap2 = -self.ky[:, None] ** 2 + self.kz2[None, :]
        self.ilap2 = 1.0 / np.where(self.lap2 == 0, 1.0, self.lap2)
        z0 = (self.ky == 0)
        self.lap2[z0, 0] = 0.0
        self.ilap2[z0, 0] = 1.0

    # spectral (dealiased, last axis) -> real z, unnormalised backward transform
    def inv(self, a):
        full = np.zeros(a.shape[:-1] + (self.NZ,), dtype=np.complex128)
        full[..., self.idx] = a
        return np.fft.ifft(full, axis=-1) * self.NZ

    def fwd(self, a):
        return np.fft.fft(a, axis=-1)[..., self.idx]

    def kxt(self, kx0, t):
        return kx0 + self.p.q * t * self.ky

    def rhs(self, t, dt_lin, lin, mf, kx0):
        p = self.p
        fac = 1.0 / self.NZ
        kx = self.kxt(kx0, t)[:, None]
        ky = self.ky[:, None]
        kz = self.kz[None, :]
        # purely imaginary wavenumbers: i*kx, i*ky, i*kz
        Kx, Ky, Kz = 1j * kx, 1j * ky, 1j * kz
        lapF = -kx * kx + self.lap2
        ilapF = 1.0 / np.where(lapF == 0, 1.0, lapF)
        mean = (self.kxi == 0) & (self.kyi == 0)
        ilapF[mean, 0] = 1.0
        il2 = self.ilap2
        u, ze, b, et = lin[:, 0], lin[:, 1], lin[:, 2], lin[:, 3]
        uy = (-Ky * Kx * u + Kz * ze) * il2
        uz = (-Kx * Kz * u - Ky * ze) * il2
        by = (-Ky * Kx * b + Kz * et) * il2
        bz = (-Kx * Kz * b - Ky * et) * il2
        F = np.zeros_like(lin)
        if p.model == 0:
            Omega = 2.0 / 3.0 * p.q
            By = self.inv(mf[1] * fac)
            dBy = self.inv(1j * self.kz * mf[1] * fac)
            ddBy = self.inv(self.kz2 * mf[1] * fac)
            Ru, Rz, Rb, Re = self.inv(u * fac), self.inv(ze * fac), self.inv(b * fac), self.inv(et * fac)
            Ruz, Rbz = self.inv(uz * fac), self.inv(bz * fac)
            Rdzuz = self.inv(Kz * uz * fac)
            F[:, 0] = self.fwd(Ky * Rb * By) + (-2 * Kx * Ky * p.q * u + 2 * Omega * Kz * ze
                                                  + self.fwd(-2 * Kx * Ky * Rbz * dBy)) * ilapF
            F[:, 1] = self.fwd(Ky * Re * By - Kx * Rb * dBy + Rbz * ddBy) + (p.q - 2 * Omega) * Kz * u
            F[:, 2] = self.fwd(Ky * Ru * By)
            F[:, 3] = self.fwd(Ky * Rz * By - (2 * Rdzuz + Kx * Ru) * dBy - Ruz * ddBy) - p.q * Kz * b
            mult = np.where(self.ky == 0, 1.0, 2.0)[:, None]
            Ruy, Rby = self.inv(uy * fac), self.inv(by * fac)
            ex = (mult * (np.real(Rbz * np.conj(Ru)) - np.real(Ruz * np.conj(Rb)))).sum(0)
            ey = (mult * (np.real(Rbz * np.conj(Ruy)) - np.real(Ruz * np.conj(Rby)))).sum(0)
            EX = 1j * self.kz * self.fwd(ex.astype(np.complex128)) * self.rs_fac
            EY = 1j * self.kz * self.fwd(ey.astype(np.complex128)) * self.rs_fac
            Fmf = np.zeros_like(mf)
            if p.quasilinear:
                Fmf[0] = EX
                Fmf[1] = -p.q * mf[0] + EY
            kxl = (kx + p.q * dt_lin * ky)
            L0 = p.nu * ((-kxl * kxl - ky * ky) + self.kz2[None, :])
            L = np.stack([L0, L0, (p.eta / p.nu) * L0, (p.eta / p.nu) * L0], axis=1)
            return F, Fmf, L
        # MHD_FullQlin
        Omega, B0z = p.omega, p.B0z
        M = [self.inv(mf[m] * fac).real for m in range(4)]
        dM = [self.inv(1j * self.kz * mf[m] * fac).real for m in range(4)]
        MBx, MBy, MUx, MUy = M
        dMBx, dMBy, dMUx, dMUy = dM
        Ux, Uy, Uz = self.inv(u * fac), self.inv(uy * fac), self.inv(uz * fac)
        Bx, By_, Bz = self.inv(b * fac), self.inv(by * fac), self.inv(bz * fac)
        # Advection by mean U along x,y: (kx MUx + ky MUy) with i, derivatives are i k f
        adv_u = Kx * MUx + Ky * MUy
        adv_b = Kx * MBx + Ky * MBy
        T1 = self.fwd(adv_u * Ux + Uz * dMUx - (adv_b * Bx + Bz * dMBx))
        T2 = self.fwd(adv_u * Uy + Uz * dMUy - (adv_b * By_ + Bz * dMBy))
        T3 = self.fwd(adv_u * Uz - adv_b * Bz)
        F[:, 0] = (-2 * Kx * Ky * p.q * u + 2 * Omega * Kz * ze + Kx * Kx * T1 + Kx * Ky * T2 + Kx * Kz * T3) * ilapF \
            + B0z * Kz * b - T1
        F[:, 1] = (p.q - 2 * Omega) * Kz * u + B0z * Kz * et - (Kz * T2 - Ky * T3)
        S1 = self.fwd(adv_u * Bx + Uz * dMBx - (adv_b * Ux + Bz * dMUx))
        S2 = self.fwd(adv_u * By_ + Uz * dMBy - (adv_b * Uy + Bz * dMUy))
        S3 = self.fwd(adv_u * Bz - adv_b * Uz)
        F[:, 2] = B0z * Kz * u - S1
        F[:, 3] = -p.q * Kz * b + B0z * Kz * ze - (Kz * S2 - Ky * S3)
        mult = np.where(self.ky == 0, 1.0, 2.0)[:, None]
        R = np.real
        cj = np.conj
        dUx, dBx = self.inv(Kz * u * fac), self.inv(Kz * b * fac)
        dUy, dBy = self.inv(Kz * uy * fac), self.inv(Kz * by * fac)
        sx = (mult * (R(Bz * cj(Ux)) - R(Uz * cj(Bx)))).sum(0)
        sy = (mult * (R(Bz * cj(Uy)) - R(Uz * cj(By_)))).sum(0)
        sux = (mult * (-(R(Ux * cj(Kx * Ux)) + R(Uy * cj(Ky * Ux)) + R(Uz * cj(dUx)))
                       + (R(Bx * cj(Kx * Bx)) + R(By_ * cj(Ky * Bx)) + R(Bz * cj(dBx))))).sum(0)
        suy = (mult * (-(R(Ux * cj(Kx * Uy)) + R(Uy * cj(Ky * Uy)) + R(Uz * cj(dUy)))
                       + (R(Bx * cj(Kx * By_)) + R(By_ * cj(Ky * By_)) + R(Bz * cj(dBy))))).sum(0)
        D = [1j * self.kz * self.fwd(sx + 0j) * self.rs_fac, 1j * self.kz * self.fwd(sy + 0j) * self.rs_fac,
             self.fwd(sux + 0j) * self.rs_fac, self.fwd(suy + 0j) * self.rs_fac]
        Fmf = np.zeros_like(mf)
        Kzr = 1j * self.kz
        if p.quasilinear:
            Fmf[1] = -p.q * mf[0] + B0z * Kzr * mf[3] + D[1]
            Fmf[0] = B0z * Kzr * mf[2] + D[0]
            Fmf[2] = 2 * Omega * mf[3] + B0z * Kzr * mf[0] + D[2]
            Fmf[3] = (p.q - 2 * Omega) * mf[2] + B0z * Kzr * mf[1] + D[3]
        kxl = (kx + p.q * dt_lin * ky)
        lf = -np.abs((-kxl * kxl - ky * ky) + self.kz2[None, :]) ** (p.viscosity_order // 2)
        L = np.stack([p.nu * lf, p.nu * lf, p.eta * lf, p.eta * lf], axis=1)
        return F, Fmf, L

    def linop_init(self, t0, kx0):
        p = self.p
        kx = self.kxt(kx0, t0)[:, None]
        lapF = -kx * kx + self.lap2
        if p.model == 0:
            L0 = p.nu * lapF
            L2 = (p.eta / p.nu) * L0
        else:
            lf = -np.abs(lapF) ** (p.viscosity_order // 2)
            L0, L2 = p.nu * lf, p.eta * lf
        Lf = np.stack([L0, L0, L2, L2], axis=1)
        coefs = [p.eta, p.eta, p.nu, p.nu][: p.nmf]
        Lm = np.stack([c * self.kz2 for c in coefs]) if p.quasilinear else np.zeros((p.nmf, self.nz))
        return Lf, Lm

    def step(self, t, lin, mf, kx0, Lold=None):
        """One RK3 step (exponential or CN per p.integrator).  Returns (lin, mf, Lold)."""
        p = self.p
        dt = p.dt
        a = [8 / 15, 5 / 12, 3 / 4]
        b = [0.0, -17 / 60, -5 / 12]
        ts = [t, t + dt * 8 / 15, t + dt * 2 / 3]
        dl = [dt * 8 / 15, dt * (2 / 3 - 8 / 15), dt * (1 - 2 / 3)]
        Lf0, Lm = self.linop_init(t, kx0)
        if Lold is None:
            Lold = Lf0
        Fp = Fpm = None
        for s in range(3):
            F, Fm, L = self.rhs(ts[s], dl[s], lin, mf, kx0)
            if p.integrator == 0:
                c = dt * (a[s] + b[s])
                acc = a[s] * dt * F + lin + (b[s] * dt * Fp if s else 0)
                accm = a[s] * dt * Fm + mf + (b[s] * dt * Fpm if s else 0)
                lin = np.exp(c * L) * acc
                mf = np.exp(c * Lm) * accm
            else:
                c = dt / 2 * (a[s] + b[s])
                den = 1.0 / (1.0 - c * L)
                denm = 1.0 / (1.0 - c * Lm)
                lin = a[s] * dt * den * F + (b[s] * dt * den * Fp if s else 0) + (1 + c * Lold) * den * lin
                mf = a[s] * dt * denm * Fm + (b[s] * dt * denm * Fpm if s else 0) + (1 + c * Lm) * denm * mf
                Lold = L
            Fp, Fpm = F, Fm
        return lin, mf, Lold

    def diagnostics(self, t, lin, mf, kx0):
        p = self.p
        kx = self.kxt(kx0, t)[:, None]
        lapF = -kx * kx + self.lap2
        l2 = lapF * self.ilap2
        mult = np.where(self.ky == 0, 1.0, 2.0)[:, None]
        n2 = lambda x: np.abs(x) ** 2
        u, ze, b, et = lin[:, 0], lin[:, 1], lin[:, 2], lin[:, 3]
        Kx, Ky, Kz = 1j * kx, 1j * self.ky[:, None], 1j * self.kz[None, :]
        uy = (-Ky * Kx * u + Kz * ze) * self.ilap2
        by = (-Ky * Kx * b + Kz * et) * self.ilap2
        Ny = p.ny // 2 * 2
        divfac = p.L[2] / float(p.nx * Ny * p.NZ) ** 2
        eu = (mult * (l2 * n2(u) - self.ilap2 * n2(ze))).sum() * divfac
        eb = (mult * (l2 * n2(b) - self.ilap2 * n2(et))).sum() * divfac
        au = (mult * np.real(u * np.conj(uy))).sum() * divfac
        ab = (mult * np.real(b * np.conj(by))).sum() * divfac
        du = (mult * p.nu * (-lapF * (l2 * n2(u) - self.ilap2 * n2(ze)))).sum() * divfac
        db = (mult * p.eta * (-lapF * (l2 * n2(b) - self.ilap2 * n2(et)))).sum() * divfac
        dm = p.L[2] / p.NZ ** 2
        eMB = (n2(mf[0]) + n2(mf[1])).sum() * dm
        aMB = np.real(mf[0] * np.conj(mf[1])).sum() * dm
        dMB = p.eta * dm * (-(self.kz2 * n2(mf[0])).sum() - (self.kz2 * n2(mf[1])).sum())
        eMU = aMU = dMU = 0.0
        if p.nmf == 4:
            eMU = (n2(mf[2]) + n2(mf[3])).sum() * dm
            aMU = np.real(mf[2] * np.conj(mf[3])).sum() * dm
            dMU = p.nu * dm * (-(self.kz2 * n2(mf[2])).sum() - (self.kz2 * n2(mf[3])).sum())
        return np.array([eMU / 2, eMB / 2, eu / 2, eb / 2, aMU, aMB, au, ab, dMU, dMB, du, db])
