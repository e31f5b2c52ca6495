"""Known-answer tests of the CPU oracle itself, and an independent numpy mirror
of the Landau step (CPU, no GPU).

The reference ships no golden vectors, so the oracle is pinned here against
answers that follow from the equations alone:

* single Fourier modes decay by exactly 1/(1 + dt L kappa k^2) (TDGL,
  Multi_MEUMAPPS.f:955-1001) and 1/(1 + dt M kappa_c k^4) (the Landau
  Cahn-Hilliard form), and a concentration mode of the reference's KKS model
  with phi = 0 by exactly 1/(1 + dt M k^2) (Multi_MEUMAPPS.f:910-949);
* uniform fields stay uniform, and follow the scalar recurrence of the
  semi-implicit step at k = 0;
* the mean concentration is conserved to round-off, in both models;
* the elastic energy of a dilatational inclusion in a homogeneous cubic medium
  equals Khachaturyan's closed form (1/2) sum_k B(n_k) |theta^(k)|^2 with
  B(n) = sigma0:eps0 - n.sigma0.Omega(n).sigma0.n, evaluated with the
  Sherman-Morrison inverse of the cubic Christoffel matrix -- the route
  ModElastic.f:115-236 takes (u^ = Q^-1 R, then elener :493-691) must give it
  to round-off;
* a numpy restatement of one Landau step (numpy.fft, batched numpy.linalg
  inverses, written independently of oracle/meu_oracle.c) agrees with the
  oracle to 1e-12.
"""
import numpy as np
import pytest

from meumapps_ss_b200 import configs as CF
from meumapps_ss_b200 import params as P

from helpers import kks_case


def _grid(n):
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    return x, y, z


def _k2(n, m):
    """|a|^2 of integer mode m (the k_space kf_sq convention: Nyquist kept)."""
    a = [2 * np.pi * (mm if mm <= n // 2 else mm - n) / n for mm in m]
    return sum(t * t for t in a)


def _mode(field, m):
    """Complex amplitude of integer mode m = (mx, my, mz) of a real (nz, ny, nx) field."""
    f = np.fft.fftn(field) / field.size
    return f[m[2] % field.shape[0], m[1] % field.shape[1], m[0] % field.shape[2]]


def _linear_landau(n, dt, kappa=1.0, kappa_c=1.0, M=1.0, L=1.0, elastic=P.ELAST_NONE):
    return CF.landau_params(n, 1, [[0.01, 0.01, 0.01]], dt=dt, A=0.0, B=0.0, Cq=0.0, D=0.0, kappa_c=kappa_c,
                            kappa_eta=kappa, M=M, L=L, elastic=elastic)


@pytest.mark.parametrize("m", [(1, 0, 0), (2, 3, 1), (8, 0, 0), (5, 8, 3), (7, 7, 7)])
def test_single_mode_decay_landau(oracle, m):
    n, dt, steps = 16, 0.01, 7
    p = _linear_landau(n, dt, kappa=1.3, kappa_c=0.7, M=1.1, L=0.9)
    x, y, z = _grid(n)
    ph = 2 * np.pi * (m[0] * x + m[1] * y + m[2] * z) / n
    c = (0.3 + 0.01 * np.cos(ph + 0.4))[None]
    e = (0.02 * np.cos(ph - 1.1))[None]
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    o.run(steps)
    c1, e1, _, _ = o.get_fields()
    k2 = _k2(n, m)
    fc = (1.0 / (1.0 + dt * 1.1 * 0.7 * k2 * k2)) ** steps
    fe = (1.0 / (1.0 + dt * 0.9 * 1.3 * k2)) ** steps
    # the whole field is the decayed mode (plus the conserved mean of c)
    assert np.max(np.abs(c1[0] - (0.3 + (c[0] - 0.3) * fc))) < 1e-15
    assert np.max(np.abs(e1[0] - e[0] * fe)) < 1e-15
    assert abs(_mode(e1[0], m) / _mode(e[0], m) - fe) < 1e-12


@pytest.mark.parametrize("m", [(1, 0, 0), (3, 2, 5), (8, 8, 8)])
def test_single_mode_decay_kks_concentration(oracle, m):
    # the reference's own model: with phi = 0 every flux term p'(phi)(X_e1 - X_en) grad phi
    # vanishes and the concentration obeys the implicit k^2 update alone
    deck, p, cons, phi = kks_case(16, 1, 5, hetero=False)
    n = p.nx
    x, y, z = _grid(n)
    ph = 2 * np.pi * (m[0] * x + m[1] * y + m[2] * z) / n
    c0 = 0.15
    cons = (c0 + 0.02 * np.cos(ph + 0.3))[None]
    phi = np.zeros_like(phi)
    o = oracle.OracleSim(p)
    o.set_fields(cons, phi)
    steps = 4
    o.run(steps)
    c1, f1, _, _ = o.get_fields()
    fac = (1.0 / (1.0 + p.dt * p.cmobs[0] * _k2(n, m))) ** steps
    assert np.max(np.abs(f1)) == 0.0
    assert np.max(np.abs(c1[0] - (c0 + (cons[0] - c0) * fac))) < 1e-15


def test_uniform_fields_follow_the_k0_recurrence(oracle):
    n, dt, L = 12, 0.01, 0.8
    p = CF.landau_params(n, 2, CF.tetragonal_variants(0.02, -0.005, 2), dt=dt, L=L, cross_w=0.5,
                         elastic=P.ELAST_NONE)
    cb, eta = 0.42, np.array([0.31, -0.17])
    o = oracle.OracleSim(p)
    o.set_fields(np.full((1, n, n, n), cb), eta[:, None, None, None] * np.ones((2, n, n, n)))
    steps = 6
    o.run(steps)
    c1, e1, _, _ = o.get_fields()
    e = eta.copy()
    for _ in range(steps):
        s2 = np.sum(e * e)
        g = p.lan_b * (p.lan_c2 - cb) * e - p.lan_c * e ** 3 + p.lan_d * e ** 5 + 4 * p.cross_w * e * (s2 - e * e)
        e = e - dt * L * g
    assert np.max(np.abs(c1 - cb)) < 1e-15
    for v in range(2):
        assert np.max(np.abs(e1[v] - e[v])) < 1e-14
        assert np.ptp(e1[v]) < 1e-15


def test_uniform_fields_stay_uniform_with_elasticity(oracle):
    n = 12
    p = CF.landau_params(n, 3, CF.tetragonal_variants(0.02, -0.005, 3), dt=0.005, cross_w=0.5)
    o = oracle.OracleSim(p)
    o.set_fields(np.full((1, n, n, n), 0.2), np.array([0.3, 0.1, -0.2])[:, None, None, None] * np.ones((3, n, n, n)))
    o.run(5)
    c1, e1, _, _ = o.get_fields()
    assert np.ptp(c1) < 1e-15
    for v in range(3):
        assert np.ptp(e1[v]) < 1e-15


def test_mean_concentration_is_conserved(oracle):
    from helpers import active_landau
    p, c, e = active_landau(16, 2)
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    m0 = np.mean(c)
    o.run(20)
    c1, _, _, _ = o.get_fields()
    assert abs(np.mean(c1) - m0) < 1e-14
    deck, pk, cons, phi = kks_case(16, 1, 10)
    o = oracle.OracleSim(pk)
    o.set_fields(cons, phi)
    m0 = np.mean(cons)
    o.run(10)
    c1, _, _, _ = o.get_fields()
    assert abs(np.mean(c1) - m0) < 1e-14


# ------------------------------------------------------------ Khachaturyan B(n)
def khachaturyan_b(n_vec, c11, c12, c44, eps):
    """B(n) of a dilatational eigenstrain eps*I in a cubic medium (unit vectors n, shape (...,3)):
    sigma0 = (C11 + 2 C12) eps I, Christoffel matrix G = D + (C12 + C44) n n^T with
    D = diag(C44 + xi n_i^2), xi = C11 - C12 - 2 C44, so n.G^-1.n = q / (1 + (C12 + C44) q),
    q = sum_i n_i^2 / (C44 + xi n_i^2)."""
    s = (c11 + 2 * c12) * eps
    xi = c11 - c12 - 2 * c44
    d = c44 + xi * n_vec ** 2
    # q / (1 + beta q) with numerator and denominator multiplied by d_1 d_2 d_3, which stays
    # finite where some d_i = 0 (for 250/150/100, C44 + xi = C11 - C12 - C44 = 0 along an axis)
    num = (n_vec[..., 0] ** 2 * d[..., 1] * d[..., 2] + n_vec[..., 1] ** 2 * d[..., 0] * d[..., 2]
           + n_vec[..., 2] ** 2 * d[..., 0] * d[..., 1])
    den = d[..., 0] * d[..., 1] * d[..., 2] + (c12 + c44) * num
    return 3 * s * eps - s * s * num / den


def test_khachaturyan_closed_form_matches_christoffel_inverse():
    rng = np.random.default_rng(5)
    c11, c12, c44 = 250.0, 150.0, 100.0
    cm = CF.cubic(c11, c12, c44)
    vo = [[0, 5, 4], [5, 1, 3], [4, 3, 2]]
    for _ in range(20):
        n = rng.standard_normal(3)
        n /= np.linalg.norm(n)
        g = np.array([[sum(cm[vo[i][j], vo[k][l]] * n[j] * n[l] for j in range(3) for l in range(3))
                       for k in range(3)] for i in range(3)])
        s = (c11 + 2 * c12) * 0.01
        ref = 3 * s * 0.01 - s * s * n @ np.linalg.solve(g, n)
        assert abs(khachaturyan_b(n, c11, c12, c44, 0.01) - ref) < 1e-15


def test_inclusion_energy_matches_khachaturyan(oracle):
    n, eps = 16, 0.01
    c11, c12, c44 = 250.0, 150.0, 100.0
    p = CF.landau_params(n, 1, [[eps, eps, eps]], moduli=(c11, c12, c44))
    x, y, z = _grid(n)
    # a smooth inclusion built from modes with no Nyquist component (|m| < n/2), where the
    # discrete k-vectors of k_space are the continuum ones
    rng = np.random.default_rng(9)
    theta = 0.5 * np.ones((n, n, n))
    for m in [(1, 0, 0), (0, 2, 1), (1, 1, 1), (3, -2, 1), (2, 5, -3), (7, 1, 0), (4, 4, 6)]:
        theta += 0.06 * rng.uniform(0.5, 1.0) * np.cos(2 * np.pi * (m[0] * x + m[1] * y + m[2] * z) / n
                                                       + rng.uniform(0, 2 * np.pi))
    assert theta.min() > 0 and theta.max() < 1
    eta = np.sqrt(theta)  # eps0 = eps eta^2 I: the shape function is eta^2
    o = oracle.OracleSim(p)
    o.set_fields(np.full((1, n, n, n), 0.2), eta[None])
    d = o.run(1)
    th = np.fft.fftn(eta * eta) / n ** 3
    kk = np.stack(np.meshgrid(*(np.fft.fftfreq(n) * 2 * np.pi,) * 3, indexing="ij"), axis=-1)  # (kz, ky, kx)
    kv = kk[..., ::-1]  # (kx, ky, kz) components
    kn = np.linalg.norm(kv, axis=-1)
    nz = kn > 0
    b = np.empty(kn.shape)
    b[nz] = khachaturyan_b(kv[nz] / kn[nz][:, None], c11, c12, c44, eps)
    b[~nz] = 3 * (c11 + 2 * c12) * eps * eps  # k = 0: no relaxation (u^(0) = 0, zero mean strain)
    energy = n ** 3 * 0.5 * np.sum(b * np.abs(th) ** 2)
    assert abs(d["elen"][0] - energy) <= 1e-12 * abs(energy)


def _p_inverse(theta):
    """phi with p(phi) = phi^3 (6 phi^2 - 15 phi + 10) = theta on (0, 1), by bisection."""
    lo, hi = np.zeros_like(theta), np.ones_like(theta)
    for _ in range(64):
        mid = 0.5 * (lo + hi)
        pm = mid ** 3 * (6 * mid * mid - 15 * mid + 10)
        lo, hi = np.where(pm < theta, mid, lo), np.where(pm < theta, hi, mid)
    return 0.5 * (lo + hi)


def test_kks_inclusion_energy_matches_khachaturyan(oracle):
    # The reference's own model: one variant with a tetragonal eigenstrain in a medium whose
    # matrix and precipitate share one cubic stiffness.  eldis's fixed point then keeps the
    # zeroth order (ModElastic.f:115-236) and elener's energy (ModElastic.f:493-691),
    # summed over the grid, is Khachaturyan's 1/2 sum_k B(n_k) |theta^(k)|^2 of the shape
    # function theta = p(phi), with B(n) = eps0:C:eps0 - (sig0 n) . (n C n)^-1 . (sig0 n)
    # evaluated here with numpy, independently of the oracle's discrete Q(k)
    n = 16
    deck = P.parse_input_txt(CF.kks_input_txt(n, 1, 1, hetero=False))
    p = P.kks_params(deck)
    cons, _ = P.init_fields(deck)
    assert np.array_equal(_mat(p, "cela", 0), _mat(p, "cela", 1))
    x, y, z = _grid(n)
    rng = np.random.default_rng(4)
    theta = 0.5 * np.ones((n, n, n))
    for m in [(1, 0, 0), (0, 2, 1), (1, 1, 1), (3, -2, 1), (2, 5, -3), (6, 1, 0)]:
        theta += 0.07 * rng.uniform(0.5, 1.0) * np.cos(2 * np.pi * (m[0] * x + m[1] * y + m[2] * z) / n
                                                       + rng.uniform(0, 2 * np.pi))
    assert theta.min() > 0 and theta.max() < 1
    phi = _p_inverse(theta)
    o = oracle.OracleSim(p)
    o.set_fields(cons, phi[None])
    d = o.run(1)
    cm = _mat(p, "cela", 1)
    e0 = np.array(p.trans_ppt[0][:3])
    assert not any(p.trans_ppt[0][3:6]) and not any(p.e_mean[:])
    sig0 = cm[:3, :3] @ e0  # normal stress of the eigenstrain (the cubic C has no normal-shear part)
    w0 = e0 @ sig0
    th = np.fft.fftn(p_of(phi)) / n ** 3
    kk = np.stack(np.meshgrid(*(np.fft.fftfreq(n) * 2 * np.pi,) * 3, indexing="ij"), axis=-1)[..., ::-1]
    kn = np.linalg.norm(kk, axis=-1)
    b = np.full(kn.shape, w0)  # k = 0: no relaxation (u^(0) = 0, no applied strain)
    for idx in zip(*np.nonzero(kn > 0)):
        nv = kk[idx] / kn[idx]
        g = np.array([[sum(cm[_VO[i][j], _VO[k][l]] * nv[j] * nv[l] for j in range(3) for l in range(3))
                       for k in range(3)] for i in range(3)])
        t = sig0 * nv
        b[idx] = w0 - t @ np.linalg.solve(g, t)
    energy = n ** 3 * 0.5 * np.sum(b * np.abs(th) ** 2)
    assert abs(d["elen"][0] - energy) <= 1e-12 * abs(energy), (d["elen"][0], energy)  # measured 2e-16


def p_of(phi):
    return phi ** 3 * (6 * phi * phi - 15 * phi + 10)


# ------------------------------------------------------- numpy mirror of a step
_VO = [[0, 5, 4], [5, 1, 3], [4, 3, 2]]


def _mat(p, name, ph):
    return np.array(getattr(p, name)[ph][:]).reshape(6, 6, order="F")


def _kvecs(n):
    m = np.arange(n)
    mm = np.where(m <= n // 2, m, m - n)
    a1 = 2 * np.pi * mm / n
    b1 = np.where(2 * m == n, 0.0, a1)
    kx = np.arange(n // 2 + 1)
    ax = 2 * np.pi * kx / n
    bx = np.where(2 * kx == n, 0.0, ax)
    sh = (n, n, n // 2 + 1)
    a = [np.broadcast_to(ax[None, None, :], sh), np.broadcast_to(a1[None, :, None], sh),
         np.broadcast_to(a1[:, None, None], sh)]
    b = [np.broadcast_to(bx[None, None, :], sh), np.broadcast_to(b1[None, :, None], sh),
         np.broadcast_to(b1[:, None, None], sh)]
    hw = np.where((kx == 0) | (2 * kx == n), 1.0, 2.0)[None, None, :]
    return a, b, hw


def numpy_landau_step(p, c, eta):
    """One Landau step, restated with numpy: driving force with the cross term, homogeneous
    micro-elasticity through u^ = Q^-1 R (zeroth order) and elener, semi-implicit CH (k^4)
    and TDGL updates.  Returns (c_new, eta_new, energies)."""
    n = p.nx
    n3 = n ** 3
    V = p.nvar
    A, B, Cq, D, c1, c2, w = p.lan_a, p.lan_b, p.lan_c, p.lan_d, p.lan_c1, p.lan_c2, p.cross_w
    a, b, hw = _kvecs(n)
    fwd = lambda f: np.fft.rfftn(f) / n3  # noqa: E731
    inv = lambda k: np.fft.irfftn(k, s=(n, n, n), axes=(0, 1, 2)) * n3  # noqa: E731
    c = c[0]
    if p.eig_coupling == P.EIG_H:
        th = eta ** 3 * (6 * eta ** 2 - 15 * eta + 10)
        thp = 30 * eta ** 2 * (eta - 1) ** 2
    else:
        th, thp = eta ** 2, 2 * eta
    s2 = np.sum(eta ** 2, axis=0)
    s4 = np.sum(eta ** 4, axis=0)
    s6 = np.sum(eta ** 6, axis=0)
    fch = np.sum(0.5 * A * (c - c1) ** 2 + 0.5 * B * (c2 - c) * s2 - 0.25 * Cq * s4 + D / 6 * s6 + w * (s2 * s2 - s4))
    mu = A * (c - c1) - 0.5 * B * s2
    elgrad = np.zeros_like(eta)
    elen = 0.0
    if p.elastic == P.ELAST_HOMOG:
        trans = np.array([p.trans_ppt[v][:] for v in range(V)])
        ceff = [_mat(p, "cela", ph) for ph in range(p.numph)]
        seff = [_mat(p, "sela", ph) for ph in range(p.numph)]
        tens = lambda e6: np.array([[e6[_VO[i][j]] for j in range(3)] for i in range(3)])  # noqa: E731
        sig0 = np.array([[sum(ceff[1][ij, _VO[k][l]] * tens(trans[v])[k, l] for k in range(3) for l in range(3))
                          for ij in range(6)] for v in range(V)])
        pk = np.array([fwd(th[v]) for v in range(V)])
        S = np.einsum("vk,v...->k...", sig0, pk)  # (6, kz, ky, kx)
        R = [sum(S[_VO[i][j]] * 1j * b[j] for j in range(3)) for i in range(3)]
        Q = np.zeros(a[0].shape + (3, 3))
        for i in range(3):
            for l in range(3):
                acc = 0.0
                for j in range(3):
                    for k in range(3):
                        kpr = -(a[k] * a[k]) if k == j else -(b[k] * b[j])
                        acc = acc + ceff[1][_VO[i][j], _VO[k][l]] * kpr
                Q[..., i, l] = acc
        Q[0, 0, 0] = np.eye(3)
        Qi = np.linalg.inv(Q)
        u = [sum(Qi[..., i, j] * R[j] for j in range(3)) for i in range(3)]
        for i in range(3):
            u[i][0, 0, 0] = 0
        gu = [[inv(1j * b[j] * u[i]) for j in range(3)] for i in range(3)]  # gu[i][j] = d_j u_i
        te = np.einsum("vq,v...->q...", trans, th)
        em = np.array(p.e_mean[:])
        epsv = np.array([em[0] + gu[0][0] - te[0], em[1] + gu[1][1] - te[1], em[2] + gu[2][2] - te[2],
                         2 * em[3] + gu[2][1] + gu[1][2] - 2 * te[3], 2 * em[4] + gu[2][0] + gu[0][2] - 2 * te[4],
                         2 * em[5] + gu[0][1] + gu[1][0] - 2 * te[5]])
        psum = np.sum(th, axis=0)
        Smix = np.einsum("v...,ij->...ij", th, seff[1]) + (1 - psum)[..., None, None] * seff[0]
        Cx = np.linalg.inv(Smix)
        sig = np.einsum("...ij,j...->i...", Cx, epsv)
        elmat = 0.5 * np.einsum("i...,ij,j...->...", sig, seff[0], sig)
        elp = 0.5 * np.einsum("i...,ij,j...->...", sig, seff[1], sig)
        en = (1 - psum) * elmat
        tiny = float(np.float32(1e-9))
        for v in range(V):
            if np.sum(trans[v]) > tiny:
                en = en + elp * th[v]
                t = trans[v]
                g = sig[0] * t[0] + sig[1] * t[1] + sig[2] * t[2] + 2 * (sig[3] * t[3] + sig[4] * t[4] + sig[5] * t[5])
                elgrad[v] = thp[v] * (elmat - elp) - g * thp[v]
        elen = float(np.sum(en))
    ck = fwd(c)
    bb = b[0] ** 2 + b[1] ** 2 + b[2] ** 2
    fint = n3 * np.sum(hw * 0.5 * p.kappa_c * bb * np.abs(ck) ** 2)
    k2 = a[0] ** 2 + a[1] ** 2 + a[2] ** 2
    dm = p.dt * p.cmobs[0]
    ck = (ck - dm * k2 * fwd(mu)) / (1 + dm * p.kappa_c * k2 * k2)
    eta_new = np.empty_like(eta)
    for v in range(V):
        g = np.array(p.grad_coeff[v][:]).reshape(3, 3, order="F")
        ek = fwd(eta[v])
        q = (g[0, 0] * b[0] ** 2 + g[1, 1] * b[1] ** 2 + g[2, 2] * b[2] ** 2 + (g[0, 1] + g[1, 0]) * b[0] * b[1]
             + (g[0, 2] + g[2, 0]) * b[0] * b[2] + (g[1, 2] + g[2, 1]) * b[1] * b[2])
        fint += n3 * np.sum(hw * 0.5 * q * np.abs(ek) ** 2)
        others = s2 - eta[v] ** 2
        gv = B * (c2 - c) * eta[v] - Cq * eta[v] ** 3 + D * eta[v] ** 5 + 4 * w * eta[v] * others + elgrad[v]
        den = 1 + p.dt * p.b_mob * (g[0, 0] * a[0] ** 2 + g[1, 1] * a[1] ** 2 + g[2, 2] * a[2] ** 2
                                    + (g[0, 1] + g[1, 0]) * b[0] * b[1] + (g[1, 2] + g[2, 1]) * b[1] * b[2]
                                    + (g[2, 0] + g[0, 2]) * b[2] * b[0])
        eta_new[v] = inv((ek - p.dt * p.b_mob * fwd(gv)) / den)
    return inv(ck)[None], eta_new, {"fch": fch, "fint": fint, "elen": elen}


@pytest.mark.parametrize("case", [
    dict(nvar=1, elastic=P.ELAST_HOMOG, coupling=P.EIG_ETA2),
    dict(nvar=3, elastic=P.ELAST_HOMOG, coupling=P.EIG_ETA2),
    dict(nvar=2, elastic=P.ELAST_HOMOG, coupling=P.EIG_H),
    dict(nvar=2, elastic=P.ELAST_NONE, coupling=P.EIG_ETA2),
])
def test_numpy_mirror_of_a_landau_step(oracle, case):
    from helpers import active_landau
    p, c, e = active_landau(16, case["nvar"], elastic=case["elastic"], coupling=case["coupling"])
    p.grad_coeff[0][1] = p.grad_coeff[0][3] = 0.2  # an anisotropic gradient tensor for variant 0
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    d = o.run(1)
    co, eo, _, _ = o.get_fields()
    cm, em, en = numpy_landau_step(p, c, e)
    assert np.max(np.abs(co - cm)) < 1e-12
    assert np.max(np.abs(eo - em)) < 1e-12
    for k in ("fch", "fint", "elen"):
        assert abs(d[k][0] - en[k]) <= 1e-12 * max(1.0, abs(en[k])), k
