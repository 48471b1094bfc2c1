"""Generate the golden fixtures in tests/golden/ from an independent numpy FP64 restatement.

k-wave-swift ships no golden vectors for its solver (its parity fixtures come from
k-wave-python, which is not available here), so this script restates the reference algorithm a
second time — vectorised numpy with numpy.fft, written separately from the C++ oracle — and
stores small seeded cases (inputs + outputs). tests/test_oracle.py checks the C++ oracle against
these files; the CUDA tests then check the GPU against the oracle.

Restated from k-wave-swift (paths relative to that project):
  Sources/KWave/Solver/KSpaceFirstOrder.swift:203-907, Sources/KWave/Sensor/Recording.swift:8-168,
  Sources/KWave/PML/PML.swift:17-43, Sources/KWave/Filter/Filters.swift:203-347.

Run:  python tests/golden/make_golden.py      (rewrites tests/golden/*.npz)
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "k-wave-swift_b200"))

from kwave.shapes import makeBall, makeCartCircle, makeCircle, makeDisc, toneBurst  # noqa: E402

DIRICHLET, ADDITIVE, ADDITIVE_NC = 0, 1, 2
NONE, POWER_LAW, NO_DISPERSION, STOKES = 0, 1, 2, 3
R = dict(p=1, pMax=2, pMin=4, pRms=8, pFinal=16, ux=32, uy=64, uz=128, uMax=256, uRms=512,
         uFinal=1024, iAvg=2048)


def kvec(n, d):
    val = 1.0 / (n * d)
    cutoff = (n - 1) // 2 + 1
    f = np.concatenate([np.arange(cutoff), np.arange(-(n // 2), -(n // 2) + n - cutoff)]) * val
    return 2 * math.pi * f


def pml(n, dx, dt, c, m, alpha, stag):
    a = alpha * (c / dx)
    out = np.ones(n)
    x = np.arange(1, m + 1, dtype=float)
    if stag:
        pl, pr = (m + 0.5 - x) / m, (x + 0.5) / m
    else:
        pl, pr = (m + 1 - x) / m, x / m
    for k in range(min(m, n)):
        out[k] = math.exp(-a * dt / 2 * pl[k] ** 4)
        out[n - m + k] = math.exp(-a * dt / 2 * pr[k] ** 4)
    return out


def blackman(n):
    if n <= 1:
        return np.ones(max(n, 0))
    x = 2 * math.pi * np.arange(n) / (n - 1)
    return 0.42 - 0.5 * np.cos(x) + 0.08 * np.cos(2 * x)


def interp(r, win, radius):
    pos = np.minimum(r, radius) + radius
    i0 = np.minimum(np.floor(pos).astype(int), len(win) - 2)
    frac = pos - i0
    return np.abs(win[i0] * (1 - frac) + win[i0 + 1] * frac)


def smooth(f):
    shape = f.shape
    enl = [n if n % 2 else n + 1 for n in shape]
    L = max(enl)
    win = blackman(L)
    radius = (L - 1) / 2
    axes = [np.array([0.0]) if c <= 1 else -radius + 2 * radius * np.arange(c) / (c - 1) for c in enl]
    if f.ndim == 2:
        nx, ny = shape
        ix = (np.arange(nx) + (nx + 1) // 2) % nx
        iy = (np.arange(ny) + (ny + 1) // 2) % ny
        r = np.sqrt(axes[0][ix][:, None] ** 2 + axes[1][iy][None, :] ** 2)
        W = interp(r, win, radius)
    else:
        grids = np.meshgrid(*[axes[a][: shape[a]] for a in range(f.ndim)], indexing="ij")
        r = np.sqrt(sum(g * g for g in grids))
        w = interp(r, win, radius)
        W = np.zeros(shape)
        idx = np.ix_(*[(np.arange(n) + (n + 1) // 2) % n for n in shape])
        W[idx] = w
    out = np.real(np.fft.ifftn(W * np.fft.fftn(f)))
    src, om = np.max(np.abs(f)), np.max(np.abs(out))
    return out * (src / om if om > 0 else 1.0)


def db2neper(alpha, y):
    return 100 * alpha * (1e-6 / (2 * math.pi)) ** y / (20 * math.log10(math.e))


def simulate(case):
    dim = case["dim"]
    shape = tuple(case["shape"])
    spacing = case["spacing"]
    N = int(np.prod(shape))
    dt, nt = case["dt"], case["nt"]
    c0 = np.broadcast_to(np.asarray(case["c0"], dtype=np.float32).astype(float), shape).copy()
    rho0 = np.broadcast_to(np.asarray(case["rho0"], dtype=np.float32).astype(float), shape).copy()
    c0map, rho0map = np.size(case["c0"]) > 1, np.size(case["rho0"]) > 1
    if case.get("smooth_c0") and c0map:
        c0 = smooth(c0)
    if case.get("smooth_rho0") and rho0map:
        rho0 = smooth(rho0)
    cref = c0.max() if c0map else float(c0.flat[0])
    ks = [kvec(shape[a], spacing[a]) for a in range(dim)]
    kgrids = np.meshgrid(*ks, indexing="ij")
    kmag = np.sqrt(sum(k * k for k in kgrids))
    arg = kmag * (cref * dt / 2)
    with np.errstate(invalid="ignore", divide="ignore"):
        kappa = np.where(arg == 0, 1.0, np.sin(arg) / arg)
    skappa = np.cos(arg)

    def bshape(v, a):
        s = [1] * dim
        s[a] = -1
        return v.reshape(s)

    ddp = [bshape(1j * ks[a] * np.exp(1j * ks[a] * spacing[a] / 2), a) for a in range(dim)]
    ddn = [bshape(1j * ks[a] * np.exp(-1j * ks[a] * spacing[a] / 2), a) for a in range(dim)]
    col = [bshape(np.exp(-1j * ks[a] * spacing[a] / 2), a) for a in range(dim)]
    m, alpha = case["pml_size"], case.get("pml_alpha", 2.0)
    pm = [bshape(pml(shape[a], spacing[a], dt, cref, m, alpha, False), a) for a in range(dim)]
    pms = [bshape(pml(shape[a], spacing[a], dt, cref, m, alpha, True), a) for a in range(dim)]
    c2 = c0 * c0
    dtrho0 = dt * rho0
    dtor = []
    for a in range(dim):
        if rho0map:
            r = np.moveaxis(rho0, a, 0)
            sg = np.concatenate([0.5 * (r[:-1] + r[1:]), r[-1:]], axis=0)
            dtor.append(dt / np.moveaxis(sg, 0, a))
        else:
            dtor.append(dt / rho0)
    F, IF = np.fft.fftn, np.fft.ifftn

    def ops(mask, sig, mode, is_p):
        out = []
        if mask is None or sig is None:
            return [None] * dim
        idx = np.flatnonzero(np.asarray(mask).reshape(-1) != 0)
        if idx.size == 0:
            return [None] * dim
        sig = np.asarray(sig, dtype=np.float32).astype(float)
        sig = sig.reshape(1, -1) if sig.ndim <= 1 else sig
        for a in range(dim):
            c = c0.reshape(-1)[idx]
            if is_p:
                sc = 1 / (dim * c * c) if mode == DIRICHLET else 2 * dt / (dim * c * spacing[a])
            else:
                sc = np.ones_like(c) if mode == DIRICHLET else 2 * c * dt / spacing[a]
            out.append((idx, sig, sc, mode))
        return out

    def apply(op, f, t):
        idx, sig, sc, mode = op
        if t >= sig.shape[1]:
            return f
        vals = (sig[0, t] if sig.shape[0] == 1 else sig[:, t]) * sc
        f = f.reshape(-1).copy()
        if mode == DIRICHLET:
            f[idx] = vals
        elif mode == ADDITIVE_NC:
            f[idx] += vals
        else:
            b = np.zeros(N)
            b[idx] = vals
            f += np.real(IF(skappa * F(b.reshape(shape)))).reshape(-1)
        return f.reshape(shape)

    src = case["source"]
    pops = ops(src.get("p_mask"), src.get("p"), src.get("p_mode", ADDITIVE), True)
    usig = [src.get("ux"), src.get("uy"), src.get("uz")]
    uops = [ops(src.get("u_mask"), usig[a], src.get("u_mode", ADDITIVE), False)[a] for a in range(dim)]
    p0 = None
    if src.get("p0") is not None:
        p0 = np.asarray(src["p0"], dtype=np.float32).astype(float)
        if case.get("smooth_p0", True):
            p0 = smooth(p0)
    # absorption
    absorb = None
    if case.get("alpha_coeff") is not None and case.get("alpha_mode", NONE) != NONE:
        y = case.get("alpha_power", 1.5)
        if case["alpha_mode"] == STOKES:
            y = 2.0
        anp = np.broadcast_to(np.asarray(case["alpha_coeff"], dtype=np.float32).astype(float), shape) * db2neper(1.0, y)
        stokes = case["alpha_mode"] == STOKES or abs(y - 2) < 1e-10
        with np.errstate(divide="ignore"):
            if stokes:
                tau, n1 = -2 * anp * c0, None
            else:
                tau = -2 * anp * c0 ** (y - 1)
                n1 = np.where(kmag == 0, 0.0, kmag ** (y - 2))
            eta = n2 = None
            if not stokes and case["alpha_mode"] != NO_DISPERSION:
                eta = 2 * anp * c0 ** y * math.tan(math.pi * y / 2)
                n2 = np.where(kmag == 0, 0.0, kmag ** (y - 1))
        absorb = (tau, n1, eta, n2)
    bona = None
    if case.get("b_on_a") is not None:
        b = np.broadcast_to(np.asarray(case["b_on_a"], dtype=np.float32).astype(float), shape)
        if np.max(np.abs(b)) != 0:
            bona = b
    # sensor
    rec = case["record"]
    rp = bool(rec & (R["p"] | R["pMax"] | R["pMin"] | R["pRms"] | R["iAvg"]))
    ru = bool(rec & (R["ux"] | R["uy"] | R["uz"] | R["uMax"] | R["uRms"] | R["iAvg"]))
    sens = case.get("sensor_mask")
    sampler = None
    if sens is not None:
        sens = np.asarray(sens, dtype=np.float32)
        if sens.ndim == 2 and sens.shape[0] == dim:
            npts = sens.shape[1]
            nc = 1 << dim
            I = np.zeros((npts, nc), dtype=np.int64)
            Wt = np.zeros((npts, nc))
            for pidx in range(npts):
                i0, fr = [], []
                for a in range(dim):
                    g = float(sens[a, pidx]) / spacing[a] + float(shape[a] // 2)
                    assert 0 <= g <= shape[a] - 1
                    i0.append(int(math.floor(g)))
                    fr.append(g - math.floor(g))
                for c in range(nc):
                    flat, w = 0, 1.0
                    for a in range(dim):
                        bit = (c >> a) & 1
                        ai = min(i0[a] + bit, shape[a] - 1)
                        w *= fr[a] if bit else 1 - fr[a]
                        flat = flat * shape[a] + ai
                    I[pidx, c], Wt[pidx, c] = flat, w
            sampler = lambda f: (f.reshape(-1)[I] * Wt).sum(axis=1)  # noqa: E731
        else:
            idx = np.flatnonzero(sens.reshape(-1) != 0)
            sampler = lambda f: f.reshape(-1)[idx]  # noqa: E731
    # 2D directivity of a binary sensor (Directivity.swift:41-79): per distinct angle th, the
    # pressure filtered by W(k) in k-space (real part of the inverse), sampled at the rows of th
    psampler = sampler
    ang = case.get("directivity_angle")
    if ang is not None and dim == 2 and sampler is not None and not (sens.ndim == 2 and sens.shape[0] == dim):
        row_ang = np.asarray(ang, dtype=np.float32).astype(float).reshape(-1)[idx]
        size = case.get("directivity_size")
        size = 10 * max(spacing[0], spacing[1]) if size is None or np.isnan(size) else float(size)
        kx, ky = kgrids[0], kgrids[1]
        filters = []
        for th in sorted(set(row_ang.tolist())):
            if int(case.get("directivity_pattern", 0)) == 0:
                x = (math.cos(th) * ky - math.sin(th) * kx) * (size / 2)
                with np.errstate(invalid="ignore", divide="ignore"):
                    w = np.where(x == 0, 1.0, np.sin(math.pi * x) / (math.pi * x))
            else:
                with np.errstate(invalid="ignore", divide="ignore"):
                    w = np.where(kmag == 0, 0.0, (math.sin(th) * ky + math.cos(th) * kx) / kmag)
            filters.append((w, np.flatnonzero(row_ang == th)))

        def psampler(f):
            out = np.zeros(len(idx))
            Pk = F(f)
            for w, rows in filters:
                out[rows] = np.real(IF(Pk * w)).reshape(-1)[idx[rows]]
            return out
    p = np.zeros(shape)
    u = [np.zeros(shape) for _ in range(dim)]
    rho = [np.zeros(shape) for _ in range(dim)]
    prec, urec = [], [[] for _ in range(dim)]
    for t in range(nt):
        P = F(p)
        for a in range(dim):
            u[a] = pms[a] * (pms[a] * u[a] - dtor[a] * np.real(IF(ddp[a] * kappa * P)))
        for a in range(dim):
            if uops[a] is not None:
                u[a] = apply(uops[a], u[a], t)
        nl = (2 * sum(rho) + rho0) / rho0 if bona is not None else None
        du = []
        for a in range(dim):
            d_ = np.real(IF(ddn[a] * kappa * F(u[a])))
            du.append(d_)
            mass = dtrho0 * d_ * nl if nl is not None else dtrho0 * d_
            rho[a] = pm[a] * (pm[a] * rho[a] - mass)
        for a in range(dim):
            if pops[a] is not None:
                rho[a] = apply(pops[a], rho[a], t)
        rt = sum(rho)
        eos = rt.copy()
        if absorb is not None:
            tau, n1, eta, n2 = absorb
            divu = sum(du)
            eos = eos + (tau * np.real(IF(n1 * F(rho0 * divu))) if n1 is not None else tau * rho0 * divu)
            if eta is not None:
                eos = eos - eta * np.real(IF(n2 * F(rt)))
        if bona is not None:
            eos = eos + bona * (rt * rt) / (2 * rho0)
        p = c2 * eos
        if t == 0 and p0 is not None:
            p = p0.copy()
            rho = [p0 / c2 if dim == 1 else p0 / (dim * c2) for _ in range(dim)]
            P0 = F(p)
            u = [(dtor[a] / 2) * np.real(IF(ddp[a] * kappa * P0)) for a in range(dim)]
        if sampler is not None:
            if rp:
                prec.append(psampler(p))
            if ru:
                for a in range(dim):
                    urec[a].append(sampler(np.real(IF(col[a] * F(u[a])))))
    out = {"pFinal": p}
    names = ["x", "y", "z"]
    if sampler is not None and rp:
        P_ = np.stack(prec, axis=1)
        if rec & R["p"]:
            out["p"] = P_
        if rec & R["pMax"]:
            out["pMax"] = P_.max(axis=1)
        if rec & R["pMin"]:
            out["pMin"] = P_.min(axis=1)
        if rec & R["pRms"]:
            out["pRms"] = np.sqrt(np.mean(P_ * P_, axis=1))
    if sampler is not None and ru:
        for a in range(dim):
            U = np.stack(urec[a], axis=1)
            if rec & R["u" + names[a]]:
                out["u" + names[a]] = U
            if rec & R["uMax"]:
                out[f"u{names[a]}Max"] = U.max(axis=1)
            if rec & R["uRms"]:
                out[f"u{names[a]}Rms"] = np.sqrt(np.mean(U * U, axis=1))
            if rec & R["iAvg"] and rp:
                T = U.shape[1]
                kk = np.array([k if k <= T // 2 else k - T for k in range(T)])
                sh = np.exp(1j * 2 * math.pi * kk / T * 0.5)
                us = np.real(np.fft.ifft(sh[None, :] * np.fft.fft(U, axis=1), axis=1))
                out[f"i{names[a]}Avg"] = np.mean(P_ * us, axis=1)
    if rec & R["uFinal"]:
        for a in range(dim):
            out[f"u{names[a]}Final"] = u[a]
    return out


def cases():
    rng = np.random.default_rng(20261203)
    cs = {}
    # 1D: additive tone-burst p source + binary sensor + velocity recording, heterogeneous
    n = 64
    dx = 1e-4
    dt = 0.3 * dx / 1600.0
    m = np.zeros(n, np.float32)
    m[16] = 1
    s = np.zeros(n, np.float32)
    s[24] = 1
    s[30] = 1
    c = (1500 + 100 * rng.random(n)).astype(np.float32)
    cs["1d_source_hetero"] = dict(
        dim=1, shape=[n], spacing=[dx], dt=dt, nt=60, pml_size=8, c0=c, rho0=np.float32(1000),
        source=dict(p_mask=m, p=(toneBurst(1 / dt, 2e6, 2) * 1.0).astype(np.float32), p_mode=ADDITIVE),
        sensor_mask=s, record=R["p"] | R["pMax"] | R["pMin"] | R["pRms"] | R["ux"] | R["uMax"] | R["uRms"] | R["iAvg"] | R["uFinal"])
    # 2D IVP lossless, smoothed p0, circle sensor (SolverTests-like)
    n = 32
    cs["2d_ivp"] = dict(
        dim=2, shape=[n, n], spacing=[1e-4, 1e-4], dt=2e-8, nt=40, pml_size=8, c0=np.float32(1500),
        rho0=np.float32(1000), smooth_p0=True,
        source=dict(p0=makeDisc(n, n, radius=3)), sensor_mask=makeCircle(n, n, radius=10),
        record=R["p"] | R["pMax"] | R["pRms"])
    # 2D heterogeneous absorbing nonlinear, dirichlet + velocity sources, Cartesian sensor
    nx, ny = 36, 30
    dx = 1e-4
    c = (1500 + 80 * rng.random((nx, ny))).astype(np.float32)
    rho = (1000 + 100 * rng.random((nx, ny))).astype(np.float32)
    dt = 0.3 * dx / float(c.max())
    um = np.zeros((nx, ny), np.float32)
    um[10, 8:12] = 1
    pmk = np.zeros((nx, ny), np.float32)
    pmk[25, 20] = 1
    pmk[26, 21] = 1
    sig2 = np.stack([toneBurst(1 / dt, 1.5e6, 2), 0.5 * toneBurst(1 / dt, 1.5e6, 2)]).astype(np.float32) * 100
    cart = makeCartCircle(9e-4, 12)
    cs["2d_hetero_abs_nl"] = dict(
        dim=2, shape=[nx, ny], spacing=[dx, dx], dt=dt, nt=50, pml_size=6, c0=c, rho0=rho,
        smooth_c0=True, alpha_coeff=np.float32(0.75), alpha_power=1.5, alpha_mode=POWER_LAW,
        b_on_a=np.float32(6.0),
        source=dict(p0=makeDisc(nx, ny, radius=4) * 2.0, p_mask=pmk, p=sig2, p_mode=DIRICHLET,
                    u_mask=um, ux=(toneBurst(1 / dt, 2e6, 2) * 1e-3).astype(np.float32),
                    uy=(toneBurst(1 / dt, 1e6, 2) * 1e-3).astype(np.float32), u_mode=ADDITIVE),
        sensor_mask=cart, record=R["p"] | R["pMax"] | R["pMin"] | R["ux"] | R["uy"] | R["iAvg"])
    # 2D stokes + additive-no-correction p source
    n = 28
    cs["2d_stokes_nc"] = dict(
        dim=2, shape=[n, n], spacing=[1e-4, 1.2e-4], dt=1.8e-8, nt=45, pml_size=5,
        c0=np.float32(1520), rho0=np.float32(990), alpha_coeff=np.float32(0.5), alpha_mode=STOKES,
        source=dict(p_mask=makeDisc(n, n, radius=1), p=(toneBurst(1 / 1.8e-8, 2e6, 2)).astype(np.float32),
                    p_mode=ADDITIVE_NC),
        sensor_mask=makeCircle(n, n, radius=8), record=R["p"])
    # 3D: hetero, power law no dispersion, additive p source plane, p0 ball, binary sensor plane
    nx, ny, nz = 16, 18, 20
    dx = 1e-4
    c = np.full((nx, ny, nz), 1500, np.float32)
    c[4:9, 5:10, 6:12] = 1600
    rho = np.full((nx, ny, nz), 1000, np.float32)
    rho[8:12, 3:8, 10:15] = 1100
    dt = 0.3 * dx / 1600
    pmk = np.zeros((nx, ny, nz), np.float32)
    pmk[6:9, 7:10, 4] = 1
    sm = np.zeros((nx, ny, nz), np.float32)
    sm[:, :, 15] = 1
    cs["3d_hetero_src"] = dict(
        dim=3, shape=[nx, ny, nz], spacing=[dx, dx, dx], dt=dt, nt=24, pml_size=4, c0=c, rho0=rho,
        alpha_coeff=np.float32(0.6), alpha_power=1.3, alpha_mode=NO_DISPERSION, b_on_a=np.float32(5.0),
        smooth_p0=True,
        source=dict(p0=makeBall(nx, ny, nz, radius=2), p_mask=pmk,
                    p=(toneBurst(1 / dt, 2e6, 2) * 1e3).astype(np.float32), p_mode=ADDITIVE),
        sensor_mask=sm, record=R["p"] | R["pMax"] | R["uz"] | R["uFinal"])
    # 2D sensor directivity (ParityDirectivityTests.swift:20-81 shape): point source, a line of
    # binary sensor points whose angles take three values, both patterns
    n = 48
    dx = 1e-4
    dt = 0.3 * dx / 1500.0
    pm = np.zeros((n, n), np.float32)
    pm[14, 24] = 1
    line = np.zeros((n, n), np.float32)
    line[32, 8:40] = 1
    angles = np.zeros((n, n), np.float32)
    angles[32, 8:40] = np.float32(math.pi / 2)
    angles[32, 8:19] = np.float32(math.pi / 4)
    angles[32, 29:40] = np.float32(3 * math.pi / 4)
    for name, pat in (("2d_directivity_pressure", 0), ("2d_directivity_gradient", 1)):
        cs[name] = dict(
            dim=2, shape=[n, n], spacing=[dx, dx], dt=dt, nt=70, pml_size=8, c0=np.float32(1500),
            rho0=np.float32(1000),
            source=dict(p_mask=pm, p=(toneBurst(1 / dt, 2e6, 2) * 1.0).astype(np.float32), p_mode=ADDITIVE),
            sensor_mask=line, directivity_angle=angles, directivity_size=6e-4, directivity_pattern=pat,
            record=R["p"] | R["pMax"])
    return cs


def simulate_as(case):
    """kspaceFirstOrderAS (KSpaceFirstOrderAS.swift:19-309) in FP64 with numpy: x axial, y radial,
    fields mirrored into a 4x radial expansion (p, ux: WSWA; uy: HAHS; uy / r: HSHA), one-sided
    radial PML, uy / r divergence term on r = (j + 1/2) dy, Stokes absorption, B/A."""
    nx, ny = case["shape"]
    dx, dy = case["spacing"]
    dt, nt = case["dt"], case["nt"]
    shape = (nx, ny)
    c0 = np.broadcast_to(np.asarray(case["c0"], dtype=np.float32).astype(float), shape).copy()
    rho0 = np.broadcast_to(np.asarray(case["rho0"], dtype=np.float32).astype(float), shape).copy()
    cref = c0.max()
    nye = 4 * ny
    kx, kye = kvec(nx, dx), kvec(nye, dy)
    kmag = np.sqrt(kx[:, None] ** 2 + kye[None, :] ** 2)
    arg = kmag * (cref * dt / 2)
    with np.errstate(invalid="ignore", divide="ignore"):
        kappa = np.where(arg == 0, 1.0, np.sin(arg) / arg)
    skappa = np.cos(arg)
    ddxp = (1j * kx * np.exp(1j * kx * dx / 2))[:, None]
    ddxn = (1j * kx * np.exp(-1j * kx * dx / 2))[:, None]
    ddyk = (1j * kye)[None, :]
    ysp = np.exp(1j * kye * dy / 2)[None, :]
    ysn = np.exp(-1j * kye * dy / 2)[None, :]
    m, alpha = case["pml_size"], case.get("pml_alpha", 2.0)
    pmlx = pml(nx, dx, dt, cref, m, alpha, False)[:, None]
    pmlxs = pml(nx, dx, dt, cref, m, alpha, True)[:, None]

    def pml_r(stag):
        a = alpha * (cref / dy)
        out = np.ones(ny)
        for k in range(min(m, ny)):
            x = k + 1.0
            pos = (x + 0.5) / m if stag else x / m
            out[ny - m + k] = math.exp(-a * dt / 2 * pos ** 4)
        return out[None, :]
    pmly, pmlys = pml_r(False), pml_r(True)
    invr = (1.0 / ((np.arange(ny) + 0.5) * dy))[None, :]
    c2 = c0 * c0
    rmap = np.size(case["rho0"]) > 1

    def sg(a):
        if not rmap:
            return rho0
        r = np.moveaxis(rho0, a, 0)
        return np.moveaxis(np.concatenate([0.5 * (r[:-1] + r[1:]), r[-1:]], axis=0), 0, a)
    dtorx, dtory = dt / sg(0), dt / sg(1)
    tau = None
    if case.get("alpha_coeff") is not None and case.get("alpha_mode", NONE) != NONE:
        tau = -2 * np.broadcast_to(np.asarray(case["alpha_coeff"], dtype=np.float32).astype(float), shape) \
            * db2neper(1.0, 2.0) * c0
    bona = None
    if case.get("b_on_a") is not None:
        b = np.broadcast_to(np.asarray(case["b_on_a"], dtype=np.float32).astype(float), shape)
        bona = b if np.max(np.abs(b)) != 0 else None

    def wswa(w):
        tail = w[:, 1:][:, ::-1]
        z = np.zeros((nx, 1))
        return np.concatenate([w, z, -tail, -w, z, tail], axis=1)

    def hahs(w):
        f = w[:, ::-1]
        return np.concatenate([w, f, -w, -f], axis=1)

    def hsha(w):
        f = w[:, ::-1]
        return np.concatenate([w, -f, -w, f], axis=1)
    F, IF = np.fft.fft2, np.fft.ifft2
    src = case["source"]

    def mk(mask, sig, scale):
        if mask is None or sig is None:
            return None
        idx = np.flatnonzero(np.asarray(mask).reshape(-1) != 0)
        if idx.size == 0:
            return None
        sig = np.asarray(sig, dtype=np.float32).astype(float)
        sig = sig.reshape(1, -1) if sig.ndim <= 1 else sig
        return idx, sig, scale(c0.reshape(-1)[idx])
    pmode, umode = src.get("p_mode", ADDITIVE), src.get("u_mode", ADDITIVE)
    psrc = mk(src.get("p_mask"), src.get("p"),
              lambda c: 1 / (2 * c * c) if pmode == DIRICHLET else 2 * dt / (2 * c * dx))
    uxs = mk(src.get("u_mask"), src.get("ux"), lambda c: np.ones_like(c) if umode == DIRICHLET else 2 * c * dt / dx)
    uys = mk(src.get("u_mask"), src.get("uy"), lambda c: np.ones_like(c) if umode == DIRICHLET else 2 * c * dt / dy)

    def mat_at(s_, t):
        idx, sig, sc = s_
        if t >= sig.shape[1]:
            return None
        v = (sig[0, t] if sig.shape[0] == 1 else sig[:, t]) * sc
        b = np.zeros(nx * ny)
        b[idx] = v
        return b.reshape(shape), idx, v

    def correct(mat, mir):
        return np.real(IF(skappa * F(mir(mat))))[:, :ny]

    def usrc(s_, u, t, mir):
        if s_ is None:
            return u
        r = mat_at(s_, t)
        if r is None:
            return u
        mat, idx, v = r
        if umode == DIRICHLET:
            u = u.reshape(-1).copy()
            u[idx] = v
            return u.reshape(shape)
        if umode == ADDITIVE_NC:
            return u + mat
        return u + correct(mat, mir)

    def grads(p):
        pk = kappa * F(wswa(p))
        return np.real(IF(ddxp * pk))[:, :ny], np.real(IF(ddyk * ysp * pk))[:, :ny]
    p0 = None if src.get("p0") is None else np.asarray(src["p0"], dtype=np.float32).astype(float)
    p = np.zeros(shape)
    ux, uy, rx, ry = np.zeros(shape), np.zeros(shape), np.zeros(shape), np.zeros(shape)
    sens = np.asarray(case["sensor_mask"], dtype=np.float32)
    sidx = np.flatnonzero(sens.reshape(-1) != 0)
    prec = []
    for t in range(nt):
        gx, gy = grads(p)
        ux = pmlxs * (pmlxs * ux - dtorx * gx)
        ux = usrc(uxs, ux, t, wswa)
        uy = pmlys * (pmlys * uy - dtory * gy)
        uy = usrc(uys, uy, t, hahs)
        duxdx = np.real(IF(ddxn * kappa * F(wswa(ux))))[:, :ny]
        uyk = ddyk * F(hahs(uy)) + F(hsha(invr * uy))
        duydy = np.real(IF(kappa * ysn * uyk))[:, :ny]
        if bona is not None:
            dtr = dt * (2 * (rx + ry) + rho0)
        else:
            dtr = dt * rho0
        rx = pmlx * (pmlx * rx - dtr * duxdx)
        ry = pmly * (pmly * ry - dtr * duydy)
        if psrc is not None:
            r = mat_at(psrc, t)
            if r is not None:
                mat, idx, v = r
                if pmode == DIRICHLET:
                    rx, ry = rx.reshape(-1).copy(), ry.reshape(-1).copy()
                    rx[idx] = v
                    ry[idx] = v
                    rx, ry = rx.reshape(shape), ry.reshape(shape)
                elif pmode == ADDITIVE_NC:
                    rx, ry = rx + mat, ry + mat
                else:
                    cm = correct(mat, wswa)
                    rx, ry = rx + cm, ry + cm
        rt = rx + ry
        e = rt.copy()
        if tau is not None:
            e = e + tau * rho0 * (duxdx + duydy)
        if bona is not None:
            e = e + bona * rt * rt / (2 * rho0)
        p = c2 * e
        if t == 0 and p0 is not None:
            p = p0.copy()
            rx = p0 / (2 * c2)
            ry = p0 / (2 * c2)
            gx, gy = grads(p)
            ux, uy = dtorx / 2 * gx, dtory / 2 * gy
        prec.append(p.reshape(-1)[sidx])
    return {"p": np.stack(prec, axis=1), "pFinal": p}


def cases_as():
    """Axisymmetric cases in the shapes of ParityAxisymmetricTests.swift: IVP, additive and
    Dirichlet p sources, Stokes absorption, B/A, additive ux and uy sources."""
    nx, ny = 48, 24
    dx = 1e-4
    dt = 0.3 * dx / 1500.0
    base = dict(dim=2, shape=[nx, ny], spacing=[dx, dx], dt=dt, nt=60, pml_size=6, c0=np.float32(1500),
                rho0=np.float32(1000), axisymmetric=1, smooth_p0=False, record=R["p"] | R["pFinal"])
    mask = np.zeros((nx, ny), np.float32)
    mask[30, 0:14] = 1
    p0 = np.zeros((nx, ny), np.float32)
    p0[20:25, 0:4] = 1.0
    sm = np.zeros((nx, ny), np.float32)
    sm[16, 0:3] = 1
    sig = (toneBurst(1 / dt, 2e6, 2) * 1.0).astype(np.float32)
    cs = {}
    cs["as_ivp"] = dict(base, sensor_mask=mask, source=dict(p0=p0))
    cs["as_add"] = dict(base, sensor_mask=mask, source=dict(p_mask=sm, p=sig, p_mode=ADDITIVE))
    cs["as_dir"] = dict(base, sensor_mask=mask, source=dict(p_mask=sm, p=sig, p_mode=DIRICHLET))
    cs["as_stokes"] = dict(base, sensor_mask=mask, alpha_coeff=np.float32(0.75), alpha_power=2.0, alpha_mode=STOKES,
                           source=dict(p0=p0))
    cs["as_nl"] = dict(base, sensor_mask=mask, b_on_a=np.float32(8.0), source=dict(p0=p0 * 3e6))
    cs["as_uxs"] = dict(base, sensor_mask=mask, source=dict(u_mask=sm, ux=sig * 1e-3, u_mode=ADDITIVE))
    cs["as_uys"] = dict(base, sensor_mask=mask, source=dict(u_mask=sm, uy=sig * 1e-3, u_mode=ADDITIVE))
    rng = np.random.default_rng(20261203 + 40)
    c = (1500 + 40 * rng.standard_normal((nx, ny))).astype(np.float32)
    rho = (1000 + 30 * rng.standard_normal((nx, ny))).astype(np.float32)
    cs["as_hetero"] = dict(base, sensor_mask=mask, c0=c, rho0=rho, dt=0.3 * dx / float(c.max()),
                           source=dict(p0=p0, p_mask=sm, p=sig, p_mode=ADDITIVE))
    return cs


def main():
    only = set(sys.argv[1:])   # optional: regenerate only the named cases
    for name, case in list(cases().items()) + list(cases_as().items()):
        if only and name not in only:
            continue
        out = simulate_as(case) if case.get("axisymmetric") else simulate(case)
        flat = {}
        for k, v in case.items():
            if k == "source":
                for sk, sv in v.items():
                    flat["src_" + sk] = np.asarray(sv)
            else:
                flat["in_" + k] = np.asarray(v)
        for k, v in out.items():
            flat["out_" + k] = np.asarray(v)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **flat)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
