"""FP64 CPU oracle for the quasi-incompressible smectic-isotropic pseudo-spectral step.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may
import it.  The product path (``smaiso_quasi_b200`` and ``libquasi_gpu.so``)
never calls it and fails loudly when its CUDA library is missing.

It restates, in vectorised numpy, the time loop of ``quasi/quasi.cpp`` (the
density-varying model) and ``quasi/quasi-stb.cpp`` (the pure-smectic stability
variant).  Every function cites the reference lines it follows.  The 3-D
real-to-real transforms are FFTW's unnormalised kinds (REDFT10, REDFT01,
RODFT10, RODFT01), which ``scipy.fft.dct/dst`` with ``norm=None`` compute
by the same published definitions.

Parity pin: the reference itself cannot be built as distributed (it needs
FFTW-MPI and the MPI-2 C++ bindings, neither of which is installed).  The
recipe ``oracle/build_ref.sh`` compiles the reference's own ``quasi.cpp`` /
``quasi-stb.cpp`` translation units against ``oracle/shim`` (a restatement of
the FFTW r2r kinds and an MPI that runs ranks as threads); the fixtures in
``tests/golden`` are that binary's 17-digit dumps, and
``tests/test_oracle_pin.py`` checks this module against them.

Array layout follows the reference: ``a[i, j, k]`` with x = i (the MPI slab
axis), z = k contiguous (``quasi.cpp:550,882``).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
import scipy.fft as sfft

# ----------------------------------------------------------------------------
# Model constants
# ----------------------------------------------------------------------------


@dataclasses.dataclass
class Model:
    """Model coefficients.  Defaults are ``quasi.cpp:176-219``; ``stb()`` gives
    ``quasi-stb.cpp:170-220``.  ``ep_arg`` and ``nu_arg`` are argv[2] and argv[1]
    (``quasi.cpp:176,192``); the reference has no runtime default for them, the
    build uses ep_arg=675 (epsilon=-0.675, the one-mode coexistence value) and
    nu_arg=1."""

    variant: str = "quasi"
    nx: int = 64
    ny: int = 64
    nz: int = 128
    nu_arg: float = 1.0
    ep_arg: float = 675.0
    gamma: float = 1.0
    beta: float = 2.0
    alpha: float = 1.0
    q0: float = 1.0
    amp: float = 1.34164
    rho_0: float = 0.005
    kp: float = 0.5
    rho_m_override: float | None = None
    nw: int = 8
    dt: float = 0.001
    divv_switch: int = 200
    emulate_ranks: int = 1
    # quasi-stb only: perturbation wavenumber used by the growth-rate probe
    q_pert: float = 0.5

    @staticmethod
    def stb(**kw) -> "Model":
        """``quasi-stb.cpp:170-204``: gamma=3, beta=0.4, Amp=0.3464101615,
        rho_0=0.1, rho_m=0.5, nu=0.1*argv[1], dt=5e-4."""
        base = dict(variant="stb", gamma=3.0, beta=0.4, amp=0.3464101615,
                    rho_0=0.1, kp=0.5, rho_m_override=0.5, dt=0.0005)
        base.update(kw)
        return Model(**base)

    # derived ----------------------------------------------------------------
    @property
    def ep(self) -> float:
        return -0.001 * self.ep_arg          # quasi.cpp:187

    @property
    def nu(self) -> float:
        return self.nu_arg if self.variant == "quasi" else 0.1 * self.nu_arg  # quasi.cpp:192, stb:191

    @property
    def rho_s(self) -> float:
        return self.kp * self.amp + self.rho_0   # quasi.cpp:197

    @property
    def rho_m(self) -> float:
        if self.rho_m_override is not None:
            return self.rho_m_override           # quasi-stb.cpp:197
        return self.rho_s / 2                    # quasi.cpp:198

    @property
    def dx(self) -> float:
        return (self.nx * 2.0 * math.pi / (self.q0 * self.nw)) / self.nx   # quasi.cpp:208-209

    @property
    def dy(self) -> float:
        return (self.ny * 2.0 * math.pi / (self.q0 * self.nw)) / self.ny

    @property
    def dz(self) -> float:
        return (self.nz * 2.0 * math.pi / (self.q0 * self.nw)) / self.nz

    @property
    def scale(self) -> float:
        return 0.125 / (self.nx * self.ny * self.nz)   # quasi.cpp:219

    @property
    def n0(self) -> int:
        """Planes per emulated MPI rank (``fftw_mpi_local_size_3d``, quasi.cpp:234)."""
        return self.nx // self.emulate_ranks

    def validate(self) -> None:
        p = self.emulate_ranks
        if p < 1 or self.nx % p:
            raise ValueError("emulate_ranks must divide nx")
        if p > 1 and p % 2:
            # quasi.cpp:1074-1077,1352-1358: odd rank counts deadlock/misroute
            raise ValueError("emulate_ranks must be 1 or even")


def equilibrium_amplitude(beta: float, gamma: float) -> float:
    """One-mode coexistence amplitude A0 = sqrt(9 beta / (10 gamma)).

    With psi = A cos(q0 z) and the free energy of quasi.cpp:2021-2024 the
    averages <cos^4> = 3/8, <cos^6> = 5/16 give F(A) = -eps A^2/4 - 3 beta A^4/32
    + 5 gamma A^6/96; F = F' = 0 yields A0^2 = 9 beta/(10 gamma) (1.8 for the
    quasi defaults, matching Amp=1.34164 at quasi.cpp:194)."""
    return math.sqrt(9.0 * beta / (10.0 * gamma))


# ----------------------------------------------------------------------------
# Transforms: FFTW r2r kinds (quasi.cpp:449-495)
# ----------------------------------------------------------------------------

def _r2r(a: np.ndarray, kinds: tuple[str, str, str]) -> np.ndarray:
    """Apply one FFTW kind per axis: 'E10' REDFT10 (DCT-II), 'E01' REDFT01
    (DCT-III), 'O10' RODFT10 (DST-II), 'O01' RODFT01 (DST-III)."""
    out = a
    for axis, kind in enumerate(kinds):
        typ = 2 if kind.endswith("10") else 3
        if kind.startswith("E"):
            out = sfft.dct(out, type=typ, axis=axis, norm=None, workers=-1)
        else:
            out = sfft.dst(out, type=typ, axis=axis, norm=None, workers=-1)
    return out


def CT(a):   return _r2r(a, ("E10", "E10", "E10"))   # planCT  quasi.cpp:449
def iCT(a):  return _r2r(a, ("E01", "E01", "E01"))   # iPlanCT quasi.cpp:455
def STx(a):  return _r2r(a, ("O10", "E10", "E10"))   # planSTx quasi.cpp:461
def STy(a):  return _r2r(a, ("E10", "O10", "E10"))   # planSTy quasi.cpp:467
def STz(a):  return _r2r(a, ("E10", "E10", "O10"))   # planSTz quasi.cpp:473
def iSTx(a): return _r2r(a, ("O01", "E01", "E01"))   # iPlanSTx quasi.cpp:479
def iSTy(a): return _r2r(a, ("E01", "O01", "E01"))   # iPlanSTy quasi.cpp:485
def iSTz(a): return _r2r(a, ("E01", "E01", "O01"))   # iPlanSTz quasi.cpp:491

PLAN_KINDS = {
    "CT": ("E10", "E10", "E10"), "iCT": ("E01", "E01", "E01"),
    "STx": ("O10", "E10", "E10"), "STy": ("E10", "O10", "E10"), "STz": ("E10", "E10", "O10"),
    "iSTx": ("O01", "E01", "E01"), "iSTy": ("E01", "O01", "E01"), "iSTz": ("E01", "E01", "O01"),
}


def r2r3d(a: np.ndarray, kinds) -> np.ndarray:
    return _r2r(np.asarray(a, dtype=np.float64), tuple(kinds))


# ----------------------------------------------------------------------------
# Initial conditions (seeded, reproducible across Python and the C++ host)
# ----------------------------------------------------------------------------

_M64 = (1 << 64) - 1


def splitmix_uniform(seed: int, n: int) -> np.ndarray:
    """U[0,1) stream: u_idx = (splitmix64(seed + (idx+1)*0x9E3779B97F4A7C15) >> 11) * 2^-53.
    The C++ host (ic.cpp) computes the identical sequence."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed & _M64) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def ic_field(m: Model, kind: str = "planar", seed: int = 1234, noise: float = 1e-3,
             delta: float = 0.5, eps_h: float = 0.0, q_h: float = 0.0,
             radius_frac: float = 0.3, width_wavelengths: float = 4.0,
             amp0: float | None = None, fc_size: float = 6.0) -> np.ndarray:
    """Seeded initial psi on the reference layout.

    planar    psi = A(z) cos(q0 z), A(z) = A0/2 (1 - tanh((z - Lz/2)/w))
    undulated psi = A(z) cos(q0 z + delta sin(2 pi x/Lx) sin(2 pi y/Ly))
    interface psi = A(z - h) cos(q0 (z - h)), h(x) = eps_h cos(q_h x)
    droplet   psi = A(r) cos(q0 z), A(r) = A0/2 (1 - tanh((r - R)/w)), R = radius_frac*L
    focal_conic  the reference's own IC (quasi.cpp:543-589), no noise
    stb       psi = A cos(q0 z) + (A phi/2)cos(q0 z + Q x) - (A phi/2)cos(q0 z - Q x)
              (quasi-stb.cpp:531-552, phi = 0.1, Q = q_pert)
    w = width_wavelengths * 2 pi / q0; uniform noise in [-noise, noise) added to psi.
    """
    nx, ny, nz = m.nx, m.ny, m.nz
    a0 = equilibrium_amplitude(m.beta, m.gamma) if amp0 is None else amp0
    i = np.arange(nx)[:, None, None].astype(np.float64)
    j = np.arange(ny)[None, :, None].astype(np.float64)
    k = np.arange(nz)[None, None, :].astype(np.float64)
    x, y, z = i * m.dx, j * m.dy, k * m.dz
    lx, ly, lz = nx * m.dx, ny * m.dy, nz * m.dz
    w = width_wavelengths * 2.0 * math.pi / m.q0
    if kind == "planar":
        psi = a0 * 0.5 * (1.0 - np.tanh((z - lz / 2) / w)) * np.cos(m.q0 * z) + 0 * x + 0 * y
    elif kind == "undulated":
        psi = a0 * 0.5 * (1.0 - np.tanh((z - lz / 2) / w)) * np.cos(
            m.q0 * z + delta * np.sin(2 * math.pi * x / lx) * np.sin(2 * math.pi * y / ly))
    elif kind == "interface":
        zz = z - eps_h * np.cos(q_h * x) + 0 * y
        psi = a0 * 0.5 * (1.0 - np.tanh((zz - lz / 2) / w)) * np.cos(m.q0 * zz)
    elif kind == "droplet":
        r = np.sqrt((x - lx / 2) ** 2 + (y - ly / 2) ** 2 + (z - lz / 2) ** 2)
        big_r = radius_frac * min(lx, ly, lz)
        psi = a0 * 0.5 * (1.0 - np.tanh((r - big_r) / w)) * np.cos(m.q0 * z)
    elif kind == "focal_conic":
        return focal_conic_ic(m, fc_size=fc_size)
    elif kind == "stb":
        phi = 0.1
        amp = m.amp
        # quasi-stb.cpp:549-550 uses k*dx for z (Nx = Nz there); we use dz.
        psi = (amp * np.cos(m.q0 * k * m.dz) + (amp * phi / 2) * np.cos(m.q0 * k * m.dz + m.q_pert * x)
               - (amp * phi / 2) * np.cos(m.q0 * k * m.dz - m.q_pert * x)) + 0 * y
    else:
        raise ValueError(kind)
    psi = np.broadcast_to(psi, (nx, ny, nz)).astype(np.float64).copy()
    if noise:
        u = splitmix_uniform(seed, nx * ny * nz).reshape(nx, ny, nz)
        psi += (2.0 * u - 1.0) * noise
    return psi


def focal_conic_ic(m: Model, fc_size: float) -> np.ndarray:
    """The reference's own "new" initial condition, quasi.cpp:543-589: a
    focal-conic (hyperboloid) smectic domain of size aE = bE = argv[3] at the
    bottom of the box (k < bE + 1), amplitude Amp, no noise."""
    nx, ny, nz = m.nx, m.ny, m.nz
    mid = float(nx // 2)                       # quasi.cpp:170 (integer Nx/2)
    a_e = b_e = float(fc_size)
    i = np.arange(nx)[:, None, None].astype(np.float64)
    j = np.arange(ny)[None, :, None].astype(np.float64)
    k = np.arange(nz)[None, None, :].astype(np.float64)
    xs, ys, zs = i - mid, j - mid, k + 0 * i + 0 * j
    ds = np.sqrt(xs * xs + ys * ys) + 0 * k
    inner_out = np.sqrt(((ds - mid) / a_e) ** 2 + (zs / b_e) ** 2) > 1
    inner_val = m.amp * np.cos(m.q0 * m.dz * np.sqrt(((b_e / a_e) * (ds - mid)) ** 2 + zs * zs))
    outer_val = np.where(np.abs(zs) < b_e, m.amp * np.cos(m.q0 * zs * m.dz), 0.0)
    psi = np.where(ds < mid, np.where(inner_out, 0.0, inner_val), outer_val)
    psi = np.where(zs < b_e + 1, psi, 0.0)
    return np.ascontiguousarray(np.broadcast_to(psi, (nx, ny, nz)), dtype=np.float64)


# ----------------------------------------------------------------------------
# The time step
# ----------------------------------------------------------------------------

class QuasiOracle:
    """State and step of quasi.cpp (variant 'quasi') or quasi-stb.cpp ('stb')."""

    def __init__(self, m: Model):
        m.validate()
        self.m = m
        nx, ny, nz = m.nx, m.ny, m.nz
        lx, ly, lz = nx * m.dx, ny * m.dy, nz * m.dz
        # Wavenumbers quasi.cpp:397-431 (DST index n carries mode n+1)
        self.vqx = math.pi * np.arange(nx) / lx
        self.vqy = math.pi * np.arange(ny) / ly
        self.vqz = math.pi * np.arange(nz) / lz
        self.vsx = math.pi * (np.arange(nx) + 1) / lx
        self.vsy = math.pi * (np.arange(ny) + 1) / ly
        self.vsz = math.pi * (np.arange(nz) + 1) / lz
        QX, QY, QZ = self.vqx[:, None, None], self.vqy[None, :, None], self.vqz[None, None, :]
        SX, SY, SZ = self.vsx[:, None, None], self.vsy[None, :, None], self.vsz[None, None, :]
        self.QX, self.QY, self.QZ, self.SX, self.SY, self.SZ = QX, QY, QZ, SX, SY, SZ
        # Spectral constants quasi.cpp:875-902 / quasi-stb.cpp:840-870
        self.mq2c = QX ** 2 + QY ** 2 + QZ ** 2
        opsh = m.alpha * (m.q0 ** 2 - self.mq2c) ** 2
        self.alin = m.ep - opsh
        if m.variant == "quasi":
            self.C1 = 2.0 - m.dt * m.rho_m * self.alin
            self.C2 = 1.5 - m.dt * m.rho_m * self.alin
        else:
            self.C1 = 1.0 + (m.dt / 2) * self.alin     # quasi-stb.cpp:855
            self.C2 = 1.0 - (m.dt / 2) * self.alin     # quasi-stb.cpp:856
        mqx = SX ** 2 + QY ** 2 + QZ ** 2
        mqy = QX ** 2 + SY ** 2 + QZ ** 2
        mqz = QX ** 2 + QY ** 2 + SZ ** 2
        self.mqx, self.mqy, self.mqz = mqx, mqy, mqz
        self.CM1x, self.CM2x = m.scale / (m.nu * mqx), SX / mqx
        self.CM1y, self.CM2y = m.scale / (m.nu * mqy), SY / mqy
        self.CM1z, self.CM2z = m.scale / (m.nu * mqz), SZ / mqz
        z = lambda: np.zeros((nx, ny, nz))
        self.psi = z(); self.psiq = z(); self.psiq_old = z(); self.psi_old = z()
        self.Nl = z(); self.Nl_old = z()
        self.rho = z(); self.rhoq = z(); self.rho_old = z()      # quasi.cpp:331-333 zero-initialised
        self.velx = z(); self.vely = z(); self.velz = z()
        self.divv = z(); self.p = z(); self.df = z(); self.lap = z()
        self.dtpsi = z()
        self.nloop = 0

    # -- a14: pre-loop projection and first N, quasi.cpp:905-951 ---------------
    def set_psi(self, psi: np.ndarray) -> None:
        self.psi = np.array(psi, dtype=np.float64, copy=True)

    def init(self) -> None:
        m = self.m
        self.psiq = m.scale * CT(self.psi)                      # :907-921
        self.psi = iCT(self.psiq)                               # :924-926
        self.Nl = m.beta * self.psi ** 3 - m.gamma * self.psi ** 5   # :928-936
        self.psiq_old = self.psiq.copy()                        # :939
        self.Nl = CT(self.Nl)                                   # :944-946
        self.psi_old = self.psi.copy()                          # :948
        self.divv[...] = 0.0                                    # :950
        self.nloop = 0

    # -- shifted spectral gradients, quasi.cpp:1120-1164 -----------------------
    @staticmethod
    def _shift_grad(aq, vs_x, vs_y, vs_z):
        gx = np.zeros_like(aq); gy = np.zeros_like(aq); gz = np.zeros_like(aq)
        gx[:-1] = -vs_x[:-1] * aq[1:]          # top DST index stays 0 (quirk: :1136)
        gy[:, :-1] = -vs_y[:, :-1] * aq[:, 1:]
        gz[:, :, :-1] = -vs_z[:, :, :-1] * aq[:, :, 1:]
        return gx, gy, gz

    def step(self) -> None:
        m = self.m
        self.nloop += 1                                         # :1018
        n = self.nloop
        self.Nl_old = self.Nl.copy()                            # :1032
        # a3 prologue :1036-1057
        dfq = m.alpha * (m.q0 ** 2 - self.mq2c) * self.psiq
        lapq = -self.mq2c * dfq
        if m.variant == "stb":
            _ = iCT(2 * m.kp * (m.q0 ** 2 + self.mq2c) * self.psiq)   # quasi-stb.cpp:1012,1024 (unused)
            sh = iCT(-self.alin * self.psiq)                     # quasi-stb.cpp:1019,1036
        self.df = iCT(dfq)
        lap = iCT(lapq)
        # a4 gradients :1062-1232
        Gx, Gy, Gz = self._shift_grad(self.psiq, self.SX, self.SY, self.SZ)
        Rx, Ry, Rz = self._shift_grad(self.rhoq, self.SX, self.SY, self.SZ)
        LGx = -self.mqx * Gx
        LGy = -self.mqy * Gy
        LGz = -self.mqz * Gz
        gx, gy, gz = iSTx(Gx), iSTy(Gy), iSTz(Gz)
        rdx, rdy, rdz = iSTx(Rx), iSTy(Ry), iSTz(Rz)
        ldx, ldy, ldz = iSTx(LGx), iSTy(LGy), iSTz(LGz)
        psi = self.psi
        if m.variant == "quasi":
            # a5 density law + Gaussian filter :1237-1268
            rho = m.kp * np.sqrt(m.q0 ** 2 * psi ** 2 + gx ** 2 + gy ** 2 + gz ** 2) + m.rho_0
            self.rhoq = m.scale * CT(rho) * np.exp(-1.57 * 1.57 * self.mq2c * 8)
            rho = iCT(self.rhoq)
            # a6 divv :1273-1293
            if n > m.divv_switch:
                self.divv = -((rho - self.rho_old) / m.dt + self.velx * rdx + self.vely * rdy
                              + self.velz * rdz) / (0.5 * (rho + self.rho_old))
            self.rho_old = rho.copy()
            divvq = CT(self.divv)
            # a7 stress :1298-1330
            lap = rho * lap
            Sx = lap * gx - rho * self.df * ldx
            Sy = lap * gy - rho * self.df * ldy
            Sz = lap * gz - rho * self.df * ldz
        else:
            rho = np.ones_like(psi)                             # quasi-stb.cpp:1232
            divvq = self.divv                                   # never transformed: stays 0
            mu = sh - m.beta * psi ** 3 + m.gamma * psi ** 5    # quasi-stb.cpp:1295
            Sx = rho * mu * gx
            Sy = rho * mu * gy
            Sz = rho * mu * gz
        self.rho = rho
        self.lap = lap
        Sxq, Syq, Szq = STx(Sx), STy(Sy), STz(Sz)
        # a8 pressure :1379-1418 (Sx from plane i-1 via halo #2, correct on every rank)
        Sxs = np.zeros_like(Sxq); Sxs[1:] = Sxq[:-1]
        Sys = np.zeros_like(Syq); Sys[:, 1:] = Syq[:, :-1]
        Szs = np.zeros_like(Szq); Szs[:, :, 1:] = Szq[:, :, :-1]
        num = -(self.QX * Sxs + self.QY * Sys + self.QZ * Szs)
        with np.errstate(divide="ignore", invalid="ignore"):
            if m.variant == "stb":
                pq = m.scale * (num / self.mq2c + 1 * m.nu * divvq)   # (4/3) is integer 1, quasi-stb.cpp:1399-1400
            else:
                pq = m.scale * (num / self.mq2c)
        I = np.arange(m.nx)[:, None, None]; J = np.arange(m.ny)[None, :, None]; K = np.arange(m.nz)[None, None, :]
        if m.variant == "quasi":
            mask = (I + J + K) != 0                             # :1403
        else:
            mask = (I * J * K) > 0                              # quasi-stb.cpp:1397
        pq = np.where(mask, pq, 0.0)
        self.p = iCT(pq)
        # a9 velocity :1420-1884
        vx, vy, vz = self._velocity(Sxq, Syq, Szq, divvq)
        self.velx, self.vely, self.velz = iSTx(vx), iSTy(vy), iSTz(vz)
        # a10 divv out :1888-1900
        self.divv = iCT(m.scale * divvq)
        # a11 nonlinear term :1905-1939
        if m.variant == "quasi":
            N = (rho * (m.ep * psi - self.df + m.beta * psi ** 3 - m.gamma * psi ** 5) - lap
                 - self.velx * gx - self.vely * gy - self.velz * gz)
            if n > m.divv_switch + 1:
                N = N + self.p * m.kp * np.sqrt(rdx ** 2 + rdy ** 2 + rdz ** 2) / m.rho_s ** 2
        else:
            self.dtpsi = -rho * mu - self.velx * gx - self.vely * gy - self.velz * gz   # quasi-stb.cpp:1909
            N = m.beta * psi ** 3 - m.gamma * psi ** 5 - self.velx * gx - self.vely * gy - self.velz * gz
        self.Nl = CT(N)
        if n == 1:
            self.Nl_old = self.Nl.copy()                        # :1936-1938
        # a12 update :1944-1965
        if m.variant == "quasi":
            new = (self.C1 * self.psiq - 0.5 * self.psiq_old
                   + (m.dt / 2) * m.scale * (3.0 * self.Nl - self.Nl_old)) / self.C2
        else:
            new = (self.C1 * self.psiq + (m.dt / 2) * m.scale * (3.0 * self.Nl - self.Nl_old)) / self.C2
        self.psiq_old = self.psiq
        self.psiq = new
        self.psi_old = self.psi
        self.psi = iCT(self.psiq)
        self.gx, self.gy, self.gz = gx, gy, gz

    def _velocity(self, Sxq, Syq, Szq, divvq):
        """Staggered Stokes projection quasi.cpp:1420-1872 with its boundary
        zeros (vely/velz only for j<Ny-1, k<Nz-1; velx zero on the last x plane)
        and the halo #4 plane quirk (quasi.cpp:1641-1690): on emulated rank r>=1,
        vely/velz at the rank's first plane read Sx from the previous rank's
        FIRST plane instead of its last one."""
        m = self.m
        nx, ny, nz = m.nx, m.ny, m.nz
        vx = np.zeros_like(Sxq); vy = np.zeros_like(Sxq); vz = np.zeros_like(Sxq)
        # velx, i < nx-1
        Sy = np.zeros_like(Syq); Sy[:-1, 1:, :] = Syq[1:, :-1, :]
        Sz = np.zeros_like(Szq); Sz[:-1, :, 1:] = Szq[1:, :, :-1]
        dv = np.zeros_like(divvq); dv[:-1] = divvq[1:]
        dot = self.SX * Sxq + self.QY * Sy + self.QZ * Sz
        vx = self.CM1x * (Sxq - self.CM2x * dot + m.nu * self.SX * dv)
        vx[nx - 1] = 0.0
        # Sx shifted by -1 in x, with the halo #4 quirk
        src = np.arange(nx) - 1
        n0 = m.n0
        for r in range(1, m.emulate_ranks):
            src[r * n0] = (r - 1) * n0
        sxm = np.where((np.arange(nx) > 0)[:, None, None], Sxq[np.maximum(src, 0)], 0.0)
        # vely, j < ny-1, k < nz-1
        SxA = np.zeros_like(Sxq); SxA[:, :-1, :] = sxm[:, 1:, :]
        SzA = np.zeros_like(Szq); SzA[:, :-1, 1:] = Szq[:, 1:, :-1]
        dvy = np.zeros_like(divvq); dvy[:, :-1, :] = divvq[:, 1:, :]
        dot = self.QX * SxA + self.SY * Syq + self.QZ * SzA
        vy = self.CM1y * (Syq - self.CM2y * dot + m.nu * self.SY * dvy)
        vy[:, ny - 1, :] = 0.0
        vy[:, :, nz - 1] = 0.0
        # velz, j < ny-1, k < nz-1
        SxB = np.zeros_like(Sxq); SxB[:, :, :-1] = sxm[:, :, 1:]
        SyB = np.zeros_like(Syq); SyB[:, 1:, :-1] = Syq[:, :-1, 1:]
        dvz = np.zeros_like(divvq); dvz[:, :, :-1] = divvq[:, :, 1:]
        dot = self.QX * SxB + self.QY * SyB + self.SZ * Szq
        vz = self.CM1z * (Szq - self.CM2z * dot + m.nu * self.SZ * dvz)
        vz[:, ny - 1, :] = 0.0
        vz[:, :, nz - 1] = 0.0
        return vx, vy, vz

    # -- a13 diagnostics quasi.cpp:1969-2033 -----------------------------------
    def diagnostics(self) -> tuple[float, float, float]:
        m = self.m
        sum_a = float(np.sum(np.abs(self.psi - self.psi_old)))
        sum_b = float(np.sum(np.abs(self.psi)))
        l1 = sum_a / (m.dt * sum_b)
        dx3 = m.dx * m.dx * m.dx
        mass = float(np.sum(self.rho)) * dx3
        psi = self.psi
        energy = float(np.sum(self.rho * (-0.5 * m.ep * psi ** 2 + 0.5 * m.alpha * self.df ** 2
                                          - 0.25 * m.beta * psi ** 4 + (m.gamma / 6) * psi ** 6))) * dx3
        return l1, mass, energy

    def growth_rate(self) -> float:
        """quasi-stb.cpp:2149-2157: (psiq - psiq_old)/(dt psiq_old) at
        (i = round(Q/Vqz[1]), j = 0, k = round(q0/Vqz[1]))."""
        m = self.m
        i = int(round(m.q_pert / self.vqz[1]))
        k = int(round(m.q0 / self.vqz[1]))
        return float((self.psiq[i, 0, k] - self.psiq_old[i, 0, k]) / (m.dt * self.psiq_old[i, 0, k]))

    def field(self, name: str) -> np.ndarray:
        return {"psi": self.psi, "rho": self.rho, "vx": self.velx, "vy": self.vely, "vz": self.velz,
                "p": self.p, "divv": self.divv, "psiq": self.psiq, "psiq_old": self.psiq_old,
                "dtpsi": self.dtpsi, "df": self.df}[name]


def mid_slice(a: np.ndarray) -> np.ndarray:
    """x-z slice at j = Ny/2 in the dump order of quasi.cpp:2040-2079 (i major, k minor)."""
    return a[:, a.shape[1] // 2, :].reshape(-1)


def run(m: Model, psi0: np.ndarray, steps: int) -> QuasiOracle:
    o = QuasiOracle(m)
    o.set_psi(psi0)
    o.init()
    for _ in range(steps):
        o.step()
    return o
