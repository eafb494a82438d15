"""Complex-step reference gradient of the gauge loss (test infrastructure).

Restates the variant-H timestep of cuda_native_impl/hydro-cal-src/src/functors.cu
(CalculateFluxKernel :47-202, OSHER :570-712, QS/QF :445-511, BOUNDA :513-568
for KLAS 4, 10 :204-232 and 1 :371-392, UpdateCellKernel :717-784) in numpy
over complex128, vectorised over slots.  Every comparison, max/min, |x| and
sign is taken on real parts (the branch the real run takes); everything else
is analytic, so for a perturbation theta + i*eps*v with eps ~ 1e-30,
Im(L)/eps is the directional derivative dL/dtheta . v to rounding, with the
branch choices frozen at the real state -- the same derivative the library's
adjoint computes.  Only the boundary codes 0, 1, 4, 10 (the channel decks).

The initial state follows mesh.cpp:350-361 from a water level Z0 and the bed;
FNC = 9.81 n^2 (mesh.cpp:364).

Used by the tests only, as a checker; never by the library.
"""
from typing import Sequence, Tuple

import numpy as np

C1 = 1.7
VMIN = 0.001


def _max(a, b):
    return np.where(np.real(a) >= np.real(b), a, b)


def _min(a, b):
    return np.where(np.real(a) <= np.real(b), a, b)


def _abs(a):
    return np.where(np.real(a) < 0, -a, a)


def _sign(a):
    return np.where(np.real(a) < 0, -1.0, 1.0)


class ComplexDeck:
    """The mesh arrays of a deck (hydrob200.Deck), for the complex-step run."""

    def __init__(self, deck):
        m = deck.mesh
        self.C = m.cells
        self.dt, self.hm1, self.hm2 = m.dt, m.hm1, m.hm2
        self.per_day = m.steps_per_day - 1
        self.ndays = m.ndays
        a = deck.array
        self.nac = a("nac").reshape(-1, 4).astype(np.int64) - 1
        self.klas = a("klas").reshape(-1, 4).copy()
        self.side = a("side").reshape(-1, 4).copy()
        self.cosf = a("cosf").reshape(-1, 4).copy()
        self.sinf = a("sinf").reshape(-1, 4).copy()
        self.area = a("area").copy()
        self.qt = a("qt").reshape(m.ndays, -1).copy()
        self.dqt = a("dqt").reshape(m.ndays, -1).copy()
        self.zt = a("zt").reshape(m.ndays, -1).copy()
        self.dzt = a("dzt").reshape(m.ndays, -1).copy()
        codes = set(np.unique(self.klas).tolist())
        if not codes <= {0.0, 1.0, 4.0, 10.0}:
            raise ValueError(f"complex-step reference covers KLAS 0, 1, 4, 10; deck has {sorted(codes)}")


def _qf(h, u, v):
    return (h * u, h * u * u, h * u * v, 4.905 * h * h)


def _osher(cl, ql, qr, fil):
    """OSHER, functors.cu:570-712: the 16 cases as signed sums of the pieces
    1, 2, 3, 5, 6, 7 (each case lists its pieces in increasing order)."""
    cr = np.sqrt(9.81 * qr[0])
    fir = qr[1] - 2.0 * cr
    ua = (fil + fir) * 0.5
    ca = _abs((fil - fir) * 0.25)
    rua, rca = np.real(ua), np.real(ca)
    k2 = np.where(rca < rua, 1, np.where((rua >= 0) & (rua < rca), 2, np.where((rua >= -rca) & (rua < 0), 3,
                  np.where(rua < -rca, 4, 0))))
    ql1, qr1, rcl, rcr = np.real(ql[1]), np.real(qr[1]), np.real(cl), np.real(cr)
    k1 = np.where((ql1 < rcl) & (qr1 >= -rcr), 1, np.where((ql1 >= rcl) & (qr1 >= -rcr), 2,
                  np.where((ql1 < rcl) & (qr1 < -rcr), 3, np.where((ql1 >= rcl) & (qr1 < -rcr), 4, 0))))
    any_ = (k1 != 0) & (k2 != 0)
    p1 = any_ & ((k1 == 2) | (k1 == 4))
    p2 = any_ & np.where(k2 == 1, (k1 == 1) | (k1 == 3), (k1 == 2) | (k1 == 4))
    s2 = np.where(k2 != 1, -1.0, 1.0)
    p3 = any_ & (k2 == 2)
    p5 = any_ & (k2 == 3)
    p6 = any_ & np.where(k2 == 4, k1 <= 2, k1 >= 3)
    s6 = np.where(k2 != 4, -1.0, 1.0)
    p7 = any_ & (k1 >= 3)
    out = [np.zeros_like(ua) for _ in range(4)]

    def add(mask, sign, q):
        for i in range(4):
            out[i] = out[i] + np.where(mask, sign * q[i], 0.0)

    add(p1, 1.0, _qf(ql[0], ql[1], ql[2]))
    us = fil / 3.0
    add(p2, s2, _qf(us * us / 9.81, us, ql[2]))
    ua35 = (fil + fir) * 0.5
    fil3 = fil - ua35
    add(p3, 1.0, _qf(fil3 * fil3 / 39.24, ua35, ql[2]))
    fir5 = fir - ua35
    add(p5, 1.0, _qf(fir5 * fir5 / 39.24, ua35, qr[2]))
    f6 = np.where(p5, fir5, fir)
    us6 = f6 / 3.0
    add(p6, s6, _qf(us6 * us6 / 9.81, us6, qr[2]))
    add(p7, 1.0, _qf(qr[0], qr[1], qr[2]))
    return out


def _osher_route(hL, uL, vL, bL, hR, uR, vR, zR_, bR, cs, sn, hm1, hm2):
    """Osher inputs and epilogue from left cell L to right cell R (functors.cu:151-200)."""
    clL = np.sqrt(9.81 * hL)
    ql = (hL, uL * cs + vL * sn, vL * cs - uL * sn)
    fil = ql[1] + 2.0 * clL
    hcR = _max(hR, hm1)
    zR = _max(bR, zR_)
    qr0 = _max(zR - bL, hm1)
    ur = uR * cs + vR * sn
    ratio = _min(hcR / qr0, 1.5)
    qr1 = np.where((np.real(hcR) <= hm2) | (np.real(qr0) <= hm2), VMIN * _sign(ur), ur * ratio)
    qr2 = vR * cs - uR * sn
    fo = _osher(clL, ql, (qr0, qr1, qr2), fil)
    f1 = fo[1] + (1.0 - ratio) * hcR * ur * ur * 0.5
    return fo, f1


def step(d: ComplexDeck, H, U, V, Z, zbc, fnc, t: int):
    """One step t (kt = 1 + t % per_day, jt = t // per_day) of the state
    (H, U, V, Z) [C] complex; returns the new state."""
    C = d.C
    kt, jt = 1 + t % d.per_day, t // d.per_day
    hm1, hm2 = d.hm1, d.hm2
    pos = np.repeat(np.arange(C), 4).reshape(C, 4)
    nc = d.nac
    has = nc >= 0
    ncs = np.where(has, nc, 0)
    cs, sn = d.cosf, d.sinf
    h1, u1, v1, z1, b1 = H[pos], U[pos], V[pos], Z[pos], zbc[pos]
    hn, un, vn, zn, bn = H[ncs], U[ncs], V[ncs], Z[ncs], zbc[ncs]
    ql1 = u1 * cs + v1 * sn
    ql2 = v1 * cs - u1 * sn
    zi = _max(z1, b1 + hm1)
    hc = np.where(has, _max(hn, hm1), 0.0)
    bc = np.where(has, bn, 0.0)
    zc = np.where(has, _max(bn, zn), 0.0)
    uc = np.where(has, un, 0.0)
    vc = np.where(has, vn, 0.0)
    F = [np.zeros((C, 4), complex) for _ in range(4)]
    code = d.klas
    bnd = code != 0
    r = np.real
    # boundary slots (BOUNDA, variant H)
    cl = np.sqrt(9.81 * h1)
    fil = ql1 + 2.0 * cl
    sup = bnd & (r(ql1) > r(cl)) & (r(h1) < hm2)
    F[0] = np.where(sup, h1 * ql1, F[0])
    F[1] = np.where(sup, h1 * ql1 * ql1, F[1])
    F[2] = np.where(sup, h1 * ql1 * ql2, F[2])
    F[3] = np.where(sup, 4.905 * h1 * h1, F[3])
    sub = bnd & ~sup
    f2pre = np.where(r(ql1) > 0, h1 * ql1 * ql2, 0.0)
    k4 = sub & (code == 4)
    F[0] = np.where(k4, 0.0, F[0])
    F[1] = np.where(k4, 0.0, F[1])
    F[2] = np.where(k4, 0.0, F[2])
    F[3] = np.where(k4, 4.905 * h1 * h1, F[3])
    k10 = sub & (code == 10)
    if k10.any():
        f0 = -(d.qt[jt][pos] + d.dqt[jt][pos] * kt) / np.where(d.side > 0, d.side, 1.0)
        hb0 = h1.copy()
        hb = np.zeros_like(h1)
        live = k10.copy()
        for _ in range(20):
            w = fil - f0 / hb0
            hb_new = w * w / 39.24
            hb = np.where(live, hb_new, hb)
            conv = live & (np.abs(r(hb0) - r(hb_new)) <= 0.005)
            live = live & ~conv
            hb0 = np.where(live, hb0 * 0.5 + hb_new * 0.5, hb0)
            if not live.any():
                break
        F[0] = np.where(k10, f0, F[0])
        F[1] = np.where(k10, np.where(r(hb) <= 1.0, 0.0, f0 * f0 / np.where(r(hb) <= 1.0, 1.0, hb)), F[1])
        F[2] = np.where(k10, 0.0, F[2])
        F[3] = np.where(k10, 4.905 * hb * hb, F[3])
    k1 = sub & (code == 1)
    if k1.any():
        lev = d.zt[jt][pos] + d.dzt[jt][pos] * jt
        hb1 = _max(lev - b1, hm2)
        fial = ql1 + 6.264 * np.sqrt(h1)
        shb = np.sqrt(hb1)
        ur0 = ql1.copy()
        urb = ql1.copy()
        live = k1.copy()
        for _ in range(30):
            fiar = urb - 6.264 * shb
            dsum, ddif = fial + fiar, fial - fiar
            new = dsum * ddif * ddif / hb1 / 313.92
            urb = np.where(live, new, urb)
            conv = live & (np.abs(r(urb) - r(ur0)) <= 0.0001)
            live = live & ~conv
            ur0 = np.where(live, urb, ur0)
            if not live.any():
                break
        F[0] = np.where(k1, hb1 * urb, F[0])
        F[1] = np.where(k1, hb1 * urb * urb, F[1])
        F[2] = np.where(k1, f2pre, F[2])
        F[3] = np.where(k1, 4.905 * hb1 * hb1, F[3])
    done = bnd.copy()
    # interior chain (functors.cu:113-150)
    m = ~done & (r(h1) <= hm1) & (r(hc) <= hm1)
    done |= m
    m = ~done & (r(zi) <= r(bc))
    F[0] = np.where(m, -C1 * hc ** 1.5, F[0])
    F[1] = np.where(m, h1 * ql1 * _abs(ql1), F[1])
    F[3] = np.where(m, 4.905 * h1 * h1, F[3])
    done |= m
    m = ~done & (r(zc) <= r(b1))
    F[0] = np.where(m, C1 * h1 ** 1.5, F[0])
    F[1] = np.where(m, h1 * _abs(ql1) * ql1, F[1])
    F[2] = np.where(m, h1 * _abs(ql1) * ql2, F[2])
    done |= m
    m = ~done & (r(h1) <= hm2)
    ma = m & (r(zc) > r(zi))
    dh = _max(zc - b1, hm1)
    un_ = -C1 * np.sqrt(dh)
    F[0] = np.where(ma, dh * un_, F[0])
    F[1] = np.where(ma, dh * un_ * un_, F[1])
    F[2] = np.where(ma, dh * un_ * (vc * cs - uc * sn), F[2])
    F[3] = np.where(ma, 4.905 * h1 * h1, F[3])
    mb = m & ~ma
    F[0] = np.where(mb, C1 * h1 ** 1.5, F[0])
    F[3] = np.where(mb, 4.905 * h1 * h1, F[3])
    done |= m
    m = ~done & (r(hc) <= hm2)
    ma = m & (r(zi) > r(zc))
    dh = _max(zi - bc, hm1)
    un_ = C1 * np.sqrt(dh)
    hc1 = zc - b1
    F[0] = np.where(ma, dh * un_, F[0])
    F[1] = np.where(ma, dh * un_ * un_, F[1])
    F[2] = np.where(ma, dh * un_ * ql2, F[2])
    F[3] = np.where(ma, 4.905 * hc1 * hc1, F[3])
    mb = m & ~ma
    F[0] = np.where(mb, -C1 * hc ** 1.5, F[0])
    F[1] = np.where(mb, h1 * ql1 * ql1, F[1])
    F[3] = np.where(mb, 4.905 * h1 * h1, F[3])
    done |= m
    rest = ~done & has
    own_first = pos < nc
    direct = rest & own_first
    mirror = rest & ~own_first
    if direct.any():
        fo, f1 = _osher_route(h1, u1, v1, b1, hn, un, vn, zn, bn, cs, sn, hm1, hm2)
        F[0] = np.where(direct, fo[0], F[0])
        F[1] = np.where(direct, f1, F[1])
        F[2] = np.where(direct, fo[2], F[2])
        F[3] = np.where(direct, fo[3], F[3])
    if mirror.any():
        fo, f1 = _osher_route(hn, un, vn, bn, h1, u1, v1, z1, b1, -cs, -sn, hm1, hm2)
        za = np.sqrt(fo[3] / 4.905) + bn
        hc3 = np.where(r(za) > r(b1), za - b1, 0.0)
        F[0] = np.where(mirror, -fo[0], F[0])
        F[1] = np.where(mirror, f1, F[1])
        F[2] = np.where(mirror, fo[2], F[2])
        F[3] = np.where(mirror, 4.905 * hc3 * hc3, F[3])
    # UpdateCellKernel (variant H)
    side = d.side
    slcos, slsin = side * cs, side * sn
    wh = np.sum(side * F[0], axis=1)
    fr1 = F[1] + F[3]
    wu = np.sum(slcos * fr1 - slsin * F[2], axis=1)
    wv = np.sum(slsin * fr1 + slcos * F[2], axis=1)
    dta = d.dt / d.area
    h2 = _max(H - dta * wh, hm1)
    z2 = h2 + zbc
    wsf = fnc * np.sqrt(U * U + V * V) / H ** 0.33333
    dtw = d.dt * wsf
    u2 = (H * U - dta * wu - dtw * U) / h2
    v2 = (H * V - dta * wv - dtw * V) / h2
    u2 = np.where(r(_abs(u2)) < 15.0, u2, 15.0 * _sign(u2))
    v2 = np.where(r(_abs(v2)) < 15.0, v2, 15.0 * _sign(v2))
    shallow = (r(h2) > hm1) & (r(h2) <= hm2)
    us = np.where(r(_abs(U)) < VMIN, U, VMIN * _sign(U))
    vs = np.where(r(_abs(V)) < VMIN, V, VMIN * _sign(V))
    u2 = np.where(r(h2) <= hm1, 0.0, np.where(shallow, us, u2))
    v2 = np.where(r(h2) <= hm1, 0.0, np.where(shallow, vs, v2))
    return h2, u2, v2, z2


def initial_state(Z0, U0, V0, zbc, hm1):
    """mesh.cpp:350-361: H = Z0 - ZBC where Z0 > ZBC, else H = HM1, Z = ZBC + HM1."""
    zbc = np.asarray(zbc, complex)
    dry = np.real(Z0) <= np.real(zbc)
    H = np.where(dry, hm1, Z0 - zbc)
    Z = np.where(dry, zbc + hm1, Z0 + 0 * zbc)
    return H.astype(complex), np.asarray(U0, complex), np.asarray(V0, complex), Z.astype(complex)


def rollout(d: ComplexDeck, n, zbc, Z0, U0, V0, nsteps: int, gauges: Sequence[int] = (), obs_every: int = 0):
    """The state after nsteps steps and the gauge depths after every obs_every steps."""
    n = np.asarray(n)
    fnc = 9.81 * n * n
    zbc = np.asarray(zbc, complex)
    H, U, V, Z = initial_state(Z0, U0, V0, zbc, d.hm1)
    g = np.asarray(gauges, dtype=np.int64)
    gd = []
    for t in range(nsteps):
        H, U, V, Z = step(d, H, U, V, Z, zbc, fnc, t)
        if obs_every and (t + 1) % obs_every == 0:
            gd.append(H[g].copy())
    return (H, U, V, Z), (np.array(gd) if gd else None)


def gauge_loss(d: ComplexDeck, n, zbc, Z0, U0, V0, gauges: Sequence[int], obs: np.ndarray, obs_every: int,
               nsteps: int) -> complex:
    """L = sum over t = obs_every, 2 obs_every, ... <= nsteps of sum_g (H_t[g] - obs)^2."""
    _, gd = rollout(d, n, zbc, Z0, U0, V0, nsteps, gauges, obs_every)
    r = gd - obs[: gd.shape[0]]
    return np.sum(r * r)


def directional_derivative(d: ComplexDeck, n, zbc, Z0, U0, V0, gauges, obs, obs_every, nsteps, vn=None, vz=None,
                           eps: float = 1e-30) -> Tuple[float, float]:
    """(L, dL/d(n, zbc) . (vn, vz)) by the complex step."""
    nn = np.asarray(n, complex) + (1j * eps * vn if vn is not None else 0)
    zz = np.asarray(zbc, complex) + (1j * eps * vz if vz is not None else 0)
    L = gauge_loss(d, nn, zz, np.asarray(Z0, float), U0, V0, gauges, obs, obs_every, nsteps)
    return float(np.real(L)), float(np.imag(L) / eps)
