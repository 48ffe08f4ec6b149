"""Post-loop products of a run: S11 / input impedance and far-field patterns.

  time_to_freq       js_fdtd/src/dft.js:17-38 (runs on the GPU, FP64)
  s11                js_fdtd/src/sparameters.js:118-196 (source port reflection)
  input_impedance    Zin = V(f) / I(f) (the reference derives no Zin; the
                     MATLAB original uses the same V and I transforms,
                     matlab_codes/fdtd_solve_Ch9_ex9a_12032026.m.txt:2597-2605)
  radiated_power     js_fdtd/src/farfield.js:257-314
  directivity        js_fdtd/src/farfield.js:328-607 (vectorised over angles)
  dft_frequencies / cut_angles   js_fdtd/src/index.js:63-91
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N
from .scenario import C0, ETA0, FF_NAMES, FarFieldBox, Grid


def time_to_freq(x: np.ndarray, dt: float, freqs: np.ndarray, shift: float):
    x = np.ascontiguousarray(x, dtype=np.float64)
    f = np.ascontiguousarray(freqs, dtype=np.float64)
    re, im = np.zeros(f.size), np.zeros(f.size)
    N.check(N.lib().fdtd_dft(N.dptr(x), x.size, dt, N.dptr(f), f.size, shift, N.dptr(re), N.dptr(im)))
    return re, im


def dft_frequencies(dft: dict) -> np.ndarray:
    n = int(math.floor(dft["maxFreq"] / dft["step"]))
    return np.array([(i + 1) * dft["step"] for i in range(n)], dtype=np.float64)


def s11(V: tuple, I: tuple, Z: float) -> dict:
    Vre, Vim = V
    Ire, Iim = I
    sq = math.sqrt(Z)
    aRe = 0.5 * (Vre + Z * Ire) / sq
    aIm = 0.5 * (Vim + Z * Iim) / sq
    bRe = 0.5 * (Vre - Z * Ire) / sq
    bIm = 0.5 * (Vim - Z * Iim) / sq
    denom = aRe * aRe + aIm * aIm
    ok = denom >= 1e-300
    safe = np.where(ok, denom, 1.0)
    Sre = np.where(ok, (bRe * aRe + bIm * aIm) / safe, 0.0)
    Sim = np.where(ok, (bIm * aRe - bRe * aIm) / safe, 0.0)
    mag = np.sqrt(Sre * Sre + Sim * Sim)
    with np.errstate(divide="ignore"):
        mag_db = np.where(mag > 0, 20 * np.log10(np.where(mag > 0, mag, 1.0)), -np.inf)
    return {"re": Sre, "im": Sim, "mag_dB": mag_db, "phase_deg": np.arctan2(Sim, Sre) * 180 / math.pi}


def input_impedance(V: tuple, I: tuple) -> np.ndarray:
    return (V[0] + 1j * V[1]) / (I[0] + 1j * I[1])


def port_s11(V: np.ndarray, I: np.ndarray, dt: float, freqs: np.ndarray, Z: float = 50.0) -> dict:
    """S11 and Zin of one port from its voltage and current traces (index.js:69-71)."""
    vf = time_to_freq(V, dt, freqs, 0.0)
    jf = time_to_freq(I, dt, freqs, -dt / 2)
    out = s11(vf, jf, Z)
    out["zin"] = input_impedance(vf, jf)
    return out


def _ff(acc, name, f, n):
    re, im = acc[name]
    return re[f * n:(f + 1) * n], im[f * n:(f + 1) * n]


def radiated_power(acc: dict, g: Grid, ff: FarFieldBox) -> np.ndarray:
    ni, nj, nk = ff.ui - ff.li, ff.uj - ff.lj, ff.uk - ff.lk
    sz = {"x": nj * nk, "y": ni * nk, "z": ni * nj}
    out = np.zeros(ff.nFreq)
    terms = [("z", g.dx * g.dy, "cmyzp", "cjxzp", "cmxzp", "cjyzp", 1), ("z", g.dx * g.dy, "cmyzn", "cjxzn", "cmxzn", "cjyzn", -1),
             ("y", g.dx * g.dz, "cmxyp", "cjzyp", "cmzyp", "cjxyp", 1), ("y", g.dx * g.dz, "cmxyn", "cjzyn", "cmzyn", "cjxyn", -1),
             ("x", g.dy * g.dz, "cmzxp", "cjyxp", "cmyxp", "cjzxp", 1), ("x", g.dy * g.dz, "cmzxn", "cjyxn", "cmyxn", "cjzxn", -1)]
    for f in range(ff.nFreq):
        p = 0.0
        for ax, area, m1, j1, m2, j2, sg in terms:
            n = sz[ax]
            M1, J1, M2, J2 = (_ff(acc, a, f, n) for a in (m1, j1, m2, j2))
            p += sg * float(np.sum(area * (M1[0] * J1[0] + M1[1] * J1[1] - M2[0] * J2[0] - M2[1] * J2[1])))
        out[f] = 0.5 * p
    return out


def directivity(acc: dict, g: Grid, ff: FarFieldBox, radp: np.ndarray, theta: np.ndarray, phi: np.ndarray):
    """D_theta, D_phi [nFreq, nAngles] (farfield.js:328-607)."""
    li, lj, lk, ui, uj, uk = ff.li, ff.lj, ff.lk, ff.ui, ff.uj, ff.uk
    ni, nj, nk = ui - li, uj - lj, uk - lk
    ci, cj, ck = 0.5 * (ui + li), 0.5 * (uj + lj), 0.5 * (uk + lk)
    st, ct, sp, cp = np.sin(theta), np.cos(theta), np.sin(phi), np.cos(phi)
    dth = np.zeros((ff.nFreq, theta.size))
    dph = np.zeros((ff.nFreq, theta.size))
    jpos = (lj - 1) + np.arange(nj)
    kpos = (lk - 1) + np.arange(nk)
    ipos = (li - 1) + np.arange(ni)
    for f in range(ff.nFreq):
        k = 2 * math.pi * ff.frequencies[f] / C0
        scale = k * k / (8 * math.pi * ETA0 * radp[f])
        Nt = np.zeros(theta.size, complex)
        Np = np.zeros(theta.size, complex)
        Lt = np.zeros(theta.size, complex)
        Lp = np.zeros(theta.size, complex)

        def cplx(name, n):
            re, im = _ff(acc, name, f, n)
            return re + 1j * im

        # x faces: points (j, k)
        n = nj * nk
        yy = ((jpos[:, None] - cj + 0.5) * g.dy + 0 * kpos[None, :]).ravel()
        zz = ((kpos[None, :] - ck + 0.5) * g.dz + 0 * jpos[:, None]).ravel()
        for xface, sfx in (((ui - ci) * g.dx, "p"), ((li - ci) * g.dx, "n")):
            r = xface * (st * cp)[:, None] + yy[None, :] * (st * sp)[:, None] + zz[None, :] * ct[:, None]
            e = np.exp(1j * k * r)
            Jy, Jz, My, Mz = (cplx(a + "x" + sfx, n) for a in ("cjy", "cjz", "cmy", "cmz"))
            A = g.dy * g.dz
            Nt += (e * (Jy[None, :] * (A * ct * sp)[:, None] - Jz[None, :] * (A * st)[:, None])).sum(1)
            Np += (e * Jy[None, :] * (A * cp)[:, None]).sum(1)
            Lt += (e * (My[None, :] * (A * ct * sp)[:, None] - Mz[None, :] * (A * st)[:, None])).sum(1)
            Lp += (e * My[None, :] * (A * cp)[:, None]).sum(1)
        # y faces: points (i, k)
        n = ni * nk
        xx = ((ipos[:, None] - ci + 0.5) * g.dx + 0 * kpos[None, :]).ravel()
        zz = ((kpos[None, :] - ck + 0.5) * g.dz + 0 * ipos[:, None]).ravel()
        for yface, sfx in (((uj - cj) * g.dy, "p"), ((lj - cj) * g.dy, "n")):
            r = xx[None, :] * (st * cp)[:, None] + yface * (st * sp)[:, None] + zz[None, :] * ct[:, None]
            e = np.exp(1j * k * r)
            Jx, Jz, Mx, Mz = (cplx(a + "y" + sfx, n) for a in ("cjx", "cjz", "cmx", "cmz"))
            A = g.dx * g.dz
            Nt += (e * (Jx[None, :] * (A * ct * cp)[:, None] - Jz[None, :] * (A * st)[:, None])).sum(1)
            Np += (e * (-Jx[None, :]) * (A * sp)[:, None]).sum(1)
            Lt += (e * (Mx[None, :] * (A * ct * cp)[:, None] - Mz[None, :] * (A * st)[:, None])).sum(1)
            Lp += (e * (-Mx[None, :]) * (A * sp)[:, None]).sum(1)
        # z faces: points (i, j)
        n = ni * nj
        xx = ((ipos[:, None] - ci + 0.5) * g.dx + 0 * jpos[None, :]).ravel()
        yy = ((jpos[None, :] - cj + 0.5) * g.dy + 0 * ipos[:, None]).ravel()
        for zface, sfx in (((uk - ck) * g.dz, "p"), ((lk - ck) * g.dz, "n")):
            r = xx[None, :] * (st * cp)[:, None] + yy[None, :] * (st * sp)[:, None] + zface * ct[:, None]
            e = np.exp(1j * k * r)
            Jx, Jy, Mx, My = (cplx(a + "z" + sfx, n) for a in ("cjx", "cjy", "cmx", "cmy"))
            A = g.dx * g.dy
            Nt += (e * (Jx[None, :] * (A * ct * cp)[:, None] + Jy[None, :] * (A * ct * sp)[:, None])).sum(1)
            Np += (e * (-Jx[None, :] * (A * sp)[:, None] + Jy[None, :] * (A * cp)[:, None])).sum(1)
            Lt += (e * (Mx[None, :] * (A * ct * cp)[:, None] + My[None, :] * (A * ct * sp)[:, None])).sum(1)
            Lp += (e * (-Mx[None, :] * (A * sp)[:, None] + My[None, :] * (A * cp)[:, None])).sum(1)
        dth[f] = scale * np.abs(Lp + ETA0 * Nt) ** 2
        dph[f] = scale * np.abs(Lt - ETA0 * Np) ** 2
    return dth, dph


def cut_angles():
    """index.js:77-91: xy cut (theta = 90 deg) and the folded xz cut, 1-degree steps."""
    angles = np.array([i * math.pi / 180 for i in range(360)])
    th_xy = np.full(360, math.pi / 2)
    ph_xz = np.where(angles > math.pi, math.pi, 0.0)
    th_xz = np.where(angles > math.pi, 2 * math.pi - angles, angles)
    return angles, th_xy, th_xz, ph_xz


def to_db(x: np.ndarray) -> np.ndarray:
    return 10 * np.log10(np.maximum(x, 1e-10))


def farfield_cuts(acc: dict, g: Grid, ff: FarFieldBox) -> list:
    radp = radiated_power(acc, g, ff)
    angles, th_xy, th_xz, ph_xz = cut_angles()
    dth_xy, dph_xy = directivity(acc, g, ff, radp, th_xy, angles)
    dth_xz, dph_xz = directivity(acc, g, ff, radp, th_xz, ph_xz)
    out = []
    for f in range(ff.nFreq):
        out.append({"plane": "xy", "freq_GHz": ff.frequencies[f] / 1e9,
                    "dataTheta_dB": to_db(dth_xy[f]), "dataPhi_dB": to_db(dph_xy[f])})
        out.append({"plane": "xz", "freq_GHz": ff.frequencies[f] / 1e9,
                    "dataTheta_dB": to_db(dth_xz[f]), "dataPhi_dB": to_db(dph_xz[f])})
    return out


def growth_onset(x, window: int = 250, factor: float = 10.0) -> int:
    """First step at which the envelope of a port trace (max |x| over windows
    of `window` steps) exceeds `factor` times its smallest value after the
    pulse peak: where a run's late-time growth sets in (a stability
    check of long runs).  -1 when it never does."""
    x = np.abs(np.asarray(x, dtype=np.float64))
    nw = x.size // window
    if nw < 3:
        return -1
    env = x[:nw * window].reshape(nw, window).max(axis=1)
    lo = np.inf
    for w in range(int(np.argmax(env)) + 1, nw):
        lo = min(lo, env[w])
        if lo > 0 and env[w] > factor * lo:
            return w * window
    return -1


__all__ = ["time_to_freq", "growth_onset", "dft_frequencies", "s11", "input_impedance", "port_s11", "radiated_power",
           "directivity", "cut_angles", "to_db", "farfield_cuts", "FF_NAMES"]
del C
