"""An independent numpy restatement of one time step of the reference's own model
(KKS, Multi_MEUMAPPS.f:548-1106) before its first elastic step, against the oracle.

Test infrastructure only.  numpy.fft stands in for P3DFFT (f_trans = fftn / N^3,
inv_trans = unscaled inverse) and numpy.linalg.solve for the LINPACK inverse of the
interface-composition system; everything else follows the reference's statements:
the spectral gradients and kappa-Laplacians (:575-615), the interpolation and well
functions, the composition solve, Gibbs energies, chemical potentials, fluxes and
driving forces (:634-845, constant rows of the system at :426-448), the n_tilda
projection (:824-841), the semi-implicit concentration and TDGL updates (:910-1001) and
the clip (:1008-1043).  Elasticity stays off (step < elastep0: el_grad = 0, :846-872),
noise too (step > noise_step).
"""
import numpy as np
import pytest

from meumapps_ss_b200 import configs as CF
from meumapps_ss_b200 import params as P


def _kspace(nz, ny, nx):
    """(a_d, b_d) broadcast to (nz, ny, nx) for d = x, y, z: a = 2 pi m / N with m in
    (-N/2, N/2]; b = a except at the Nyquist index, where it is 0 (k_space)."""
    out = []
    for n, ax in ((nx, 2), (ny, 1), (nz, 0)):
        m = np.arange(n)
        mm = np.where(m <= n // 2, m, m - n)
        a = 2 * np.pi * mm / n
        b = np.where(2 * m == n, 0.0, a)
        shape = [1, 1, 1]
        shape[ax] = n
        out.append((a.reshape(shape), b.reshape(shape)))
    return out  # [(ax, bx), (ay, by), (az, bz)]


def numpy_kks_step(p, cons, phi):
    """One KKS step of fields cons (numel, nz, ny, nx), phi (vartot, nz, ny, nx); returns
    the new fields and the step's energies (f_int, fw, fch)."""
    numel, numph, V = p.numel, p.numph, p.nvar
    nz, ny, nx = phi.shape[1:]
    n3 = nx * ny * nz
    (ax, bx), (ay, by), (az, bz) = _kspace(nz, ny, nx)
    kf = [1j * bx, 1j * by, 1j * bz]
    kf_sq = [-(ax * ax), -(ay * ay), -(az * az)]

    def g(v, i, j):  # grad_coeff(i, j, v), 1-based i, j
        return p.grad_coeff[v][(j - 1) * 3 + (i - 1)]

    def kdel(v):
        return (g(v, 1, 1) * kf_sq[0] + g(v, 2, 2) * kf_sq[1] + g(v, 3, 3) * kf_sq[2]
                + (g(v, 1, 2) + g(v, 2, 1)) * kf[0] * kf[1] + (g(v, 2, 3) + g(v, 3, 2)) * kf[1] * kf[2]
                + (g(v, 3, 1) + g(v, 1, 3)) * kf[2] * kf[0])

    def ftr(a):
        return np.fft.fftn(a) / n3

    def itr(a):
        return np.real(np.fft.ifftn(a) * n3)

    grads = np.empty((V, 3, nz, ny, nx))
    kdsq = np.empty((V, nz, ny, nx))
    for v in range(V):
        ph = ftr(phi[v])
        for d in range(3):
            grads[v, d] = itr(ph * kf[d])
        kdsq[v] = itr(ph * kdel(v))

    def G(j, n):  # Gparams(j, n), 1-based
        return p.gparams[n - 1][j - 1]

    # variants of each phase (phase 1 is the matrix): 0-based index ranges
    ranges, v0 = {}, 0
    for n in range(2, numph + 1):
        ranges[n] = range(v0, v0 + p.nvar_ph[n - 1])
        v0 += p.nvar_ph[n - 1]
    Pph = np.zeros((numph,) + phi.shape[1:])
    Gph = np.zeros((numph,) + phi.shape[1:])
    Ppr = np.zeros_like(phi)
    for n in range(2, numph + 1):
        for v in ranges[n]:
            fi = phi[v]
            pl = fi ** 2 * fi * (6 * fi ** 2 - 15 * fi + 10)
            Ppr[v] = 30 * fi ** 2 * (fi ** 2 - 2 * fi + 1)
            Pph[0] += pl
            Pph[n - 1] += pl
            Gph[n - 1] += fi ** 2 * (1 - fi) ** 2
            for u in range(V):
                if u != v:
                    Gph[0] += fi ** 2 * phi[u] ** 2
    Pph[0] = 1 - Pph[0]
    # interface compositions: constant rows (:426-448), per-voxel rows (:677-688)
    zdim = numph * numel
    nv = n3
    Z = np.zeros((nv, zdim, zdim))
    Zr = np.zeros((nv, zdim))
    for e in range(1, numel + 1):
        i1 = e + numel + 1
        for n in range(1, numph):
            i0 = (numph - 1) * (e - 1) + n
            j0 = numph * (e - 1) + n
            Z[:, i0 - 1, j0 - 1] = G(e, n)
            Z[:, i0 - 1, j0] = -G(e, n + 1)
            Zr[:, i0 - 1] = G(e, n) * G(i1, n) - G(e, n + 1) * G(i1, n + 1)
    for e in range(1, numel + 1):
        i0 = zdim - numel + e
        Zr[:, i0 - 1] = cons[e - 1].reshape(-1)
        for n in range(1, numph + 1):
            Z[:, i0 - 1, numph * (e - 1) + n - 1] = Pph[n - 1].reshape(-1)
    Xv = np.linalg.solve(Z, Zr[..., None])[..., 0]
    X = {(e, n): Xv[:, numph * (e - 1) + n - 1].reshape(phi.shape[1:])
         for e in range(1, numel + 1) for n in range(1, numph + 1)}
    Gib = {}
    for n in range(1, numph + 1):
        acc = 0.0
        for e in range(1, numel + 1):
            acc = acc + G(e, n) * (X[e, n] - G(e + numel + 1, n)) ** 2
        Gib[n] = acc + G(numel + 1, n)
    Mu = {e: 2 * G(e, 1) * (X[e, 1] - G(e + numel + 1, 1)) for e in range(1, numel + 1)}
    fch = Pph[0] * Gib[1]
    fw = p.wellph[0] * Gph[0]
    f_int = 0.0
    Fcon = np.zeros((numel, 3) + phi.shape[1:])
    fgrad = np.zeros_like(phi)
    for n in range(2, numph + 1):
        for v in ranges[n]:
            gx, gy, gz = grads[v]
            term = (g(v, 1, 1) * gx ** 2 + g(v, 2, 2) * gy ** 2 + g(v, 3, 3) * gz ** 2
                    + (g(v, 1, 2) + g(v, 2, 1)) * gx * gy + (g(v, 1, 3) + g(v, 3, 1)) * gx * gz
                    + (g(v, 2, 3) + g(v, 3, 2)) * gy * gz)
            f_int += 0.5 * np.sum(term)
            fi = phi[v]
            termch = Gib[n] - Gib[1]
            for e in range(1, numel + 1):
                xd = X[e, 1] - X[e, n]
                termch = termch + Mu[e] * xd
                for d in range(3):
                    Fcon[e - 1, d] += Ppr[v] * xd * grads[v, d]
            well = 2 * p.wellph[n - 1] * fi * (1 - fi) * (1 - 2 * fi)
            for u in range(V):
                if u != v:
                    well = well + 4 * p.wellph[0] * fi * phi[u] ** 2
            fgrad[v] = termch * Ppr[v] + well
        fch = fch + Pph[n - 1] * Gib[n]
        fw = fw + p.wellph[n - 1] * Gph[n - 1]
    # n_tilda projection
    fdiff = np.empty_like(phi)
    for j in range(V):
        t11 = np.zeros(phi.shape[1:])
        nt = np.ones(phi.shape[1:])
        for i in range(V):
            if i == j:
                continue
            on = (phi[j] > 0) & (phi[i] > 0)
            t11 = t11 + np.where(on, fgrad[i] - kdsq[i], 0.0)
            nt = nt + on
        fdiff[j] = fgrad[j] - t11 / nt
    # Cahn-Hilliard (diffusion) update
    k_sq = kf_sq[0] + kf_sq[1] + kf_sq[2]
    c_new = np.empty_like(cons)
    for e in range(numel):
        t1 = sum(kf[d] * ftr(Fcon[e, d]) for d in range(3))
        t2 = 1 - p.dt * p.cmobs[e] * k_sq
        c_new[e] = itr((ftr(cons[e]) + p.dt * p.cmobs[e] * t1) / t2)
    # TDGL update, then the clip
    phi_new = np.empty_like(phi)
    for v in range(V):
        t2 = 1 - p.dt * p.b_mob * kdel(v)
        phi_new[v] = np.clip(itr((ftr(phi[v]) - p.dt * p.b_mob * ftr(fdiff[v])) / t2), 0.0, 1.0)
    return c_new, phi_new, {"fint": f_int, "fw": float(np.sum(fw)), "fch": float(np.sum(fch))}


@pytest.mark.parametrize("nvar,numel_in", [(1, 2), (3, 2), (3, 3)])
def test_numpy_mirror_of_a_kks_step(oracle, nvar, numel_in):
    # The deck's set-up (Input.txt format; 1 or 3 variants, 1 or 2 solutes) with fields that
    # exercise every branch: every variant nonzero almost everywhere (cross terms), 15%
    # exact zeros (the n_tilda projection's phi > 0 tests), values up to 1.05 (the clip),
    # solutes with noise, and nonzero energy wells (the deck's interfacial energies are 0)
    n = 16
    deck = P.parse_input_txt(CF.kks_input_txt(n, nvar, 5, elastep0=1000, numel_in=numel_in))
    p = P.kks_params(deck)
    assert p.step < p.elastep0 and p.step > p.noise_step
    for k in range(p.numph):
        p.wellph[k] = 1.0e8 * (k + 1)
    rng = np.random.default_rng(7 + nvar + numel_in)
    cons0, phi0 = P.init_fields(deck)
    phi = rng.uniform(0.0, 1.05, phi0.shape) * (rng.uniform(size=phi0.shape) > 0.15)
    cons = cons0.mean(axis=(1, 2, 3), keepdims=True) + 0.05 * rng.uniform(-1, 1, cons0.shape)
    c1, f1, en = numpy_kks_step(p, cons, phi)
    assert np.any(f1 == 1.0)  # the clip acted
    o = oracle.OracleSim(p)
    o.set_fields(cons, phi)
    d = o.run(1)
    co, fo, _, _ = o.get_fields()
    # measured: fields to 8e-16, energies to 4e-16 relative
    assert np.max(np.abs(co - c1)) <= 1e-12 * np.max(np.abs(c1))
    assert np.max(np.abs(fo - f1)) <= 1e-12
    for k in ("fint", "fw", "fch"):
        assert en[k] != 0.0
        assert abs(d[k][0] - en[k]) <= 1e-12 * abs(en[k]), (k, d[k][0], en[k])
