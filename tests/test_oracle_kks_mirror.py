"""An independent numpy restatement of one time step of the reference's own model
(KKS, Multi_MEUMAPPS.f:548-1106), against the oracle: before the first elastic step,
and at it with heterogeneous moduli (eldis and elener, ModElastic.f:105-691).

Test infrastructure only.  numpy.fft stands in for P3DFFT (f_trans = fftn / N^3,
inv_trans = unscaled inverse) and numpy.linalg.solve for the LINPACK inverse of the
interface-composition system; everything else follows the reference's statements:
the spectral gradients and kappa-Laplacians (:575-615), the interpolation and well
functions, the composition solve, Gibbs energies, chemical potentials, fluxes and
driving forces (:634-845, constant rows of the system at :426-448), the n_tilda
projection (:824-841), the semi-implicit concentration and TDGL updates (:910-1001) and
the clip (:1008-1043); at the first elastic step the zeroth order, the fixed point with
its convergence test, backtracking and cfac ramp, and elener's energy and driving force
(batched numpy.linalg inverses for Q(k) and the per-voxel compliance mixes).  Noise
stays off (step > noise_step).  Measured agreement: fields to 8e-16, energies to 3e-15
relative, the same fixed-point iteration count.
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


_VO = [[0, 5, 4], [5, 1, 3], [4, 3, 2]]  # Voigt index of (i, j), 0-based


def _mat(p, name, n):
    return np.array(getattr(p, name)[n][:]).reshape(6, 6, order="F")


def numpy_eldis(p, Pphi, phi, ranges):
    """eldis at the first elastic step (ModElastic.f:105-481: the zeroth order, then the
    fixed point with damping, backtracking and the cfac ramp) followed by elener
    (:493-691).  Returns el_en, el_grad and the iterations run."""
    V = p.nvar
    nz, ny, nx = phi.shape[1:]
    n3 = nx * ny * nz
    (ax, bx), (ay, by), (az, bz) = _kspace(nz, ny, nx)
    kf = [1j * bx, 1j * by, 1j * bz]
    kf_sq = [-(ax * ax), -(ay * ay), -(az * az)]

    def ftr(a):
        return np.fft.fftn(a) / n3

    def itr(a):
        return np.real(np.fft.ifftn(a) * n3)

    phase = {v: n for n, r in ranges.items() for v in r}
    cel = {n: _mat(p, "cela", n - 1) for n in range(1, p.numph + 1)}
    sel = {n: _mat(p, "sela", n - 1) for n in range(1, p.numph + 1)}
    tr = np.array([p.trans_ppt[v][:6] for v in range(V)])  # tensor Voigt
    em = np.array(p.e_mean[:6])
    full = np.broadcast_shapes(kf[0].shape, kf[1].shape, kf[2].shape)
    # Q(i,l) = sum_jk C2(ij,kl) kpr, kpr = kf_k kf_j (k != j) or kf_sq_k (k == j)
    Q = np.zeros(full + (3, 3), dtype=complex)
    for i in range(3):
        for j in range(3):
            for k in range(3):
                for l in range(3):
                    kpr = kf_sq[k] if k == j else kf[k] * kf[j]
                    Q[..., i, l] += cel[2][_VO[i][j], _VO[k][l]] * np.broadcast_to(kpr, full)
    Q = np.real(Q)
    k0 = (0, 0, 0)
    Q[k0] = np.eye(3)
    Qi = np.linalg.inv(Q)
    # eigenstress of each variant with its phase's stiffness, summed over all (k, l)
    sig0 = np.zeros((V, 3, 3))
    for v in range(V):
        for i in range(3):
            for j in range(3):
                sig0[v, i, j] = sum(cel[phase[v]][_VO[i][j], _VO[k][l]] * tr[v, _VO[k][l]]
                                    for k in range(3) for l in range(3))
    Ph = [ftr(Pphi[v]) for v in range(V)]

    def solve_u(Rv):
        u = [sum(Qi[..., i, m] * Rv[m] for m in range(3)) for i in range(3)]
        for i in range(3):
            u[i][k0] = 0.0
        return u

    R0 = [sum(kf[j] * sum(Ph[v] * sig0[v, i, j] for v in range(V)) for j in range(3)) for i in range(3)]
    uh = solve_u(R0)
    u = np.array([itr(uh[i]) for i in range(3)])
    gu = np.array([[itr(kf[l] * uh[k]) for l in range(3)] for k in range(3)])  # gu[k, l] = d_l u_k
    psum = sum(Pphi[v] for v in range(V))
    Cmix = np.zeros(phi.shape[1:] + (6, 6))
    for v in range(V):
        Cmix += Pphi[v][..., None, None] * sel[phase[v]]
    Cmix += np.where(psum < 1, 1 - psum, 0.0)[..., None, None] * sel[1]
    Cv = np.linalg.inv(Cmix)
    Cp = cel[2] - Cv
    newfac, niter, cfac, converged, err_old, total = 0.5, 0, 1.0, False, None, 0
    while True:
        u_old = u.copy()
        niter += 1
        total += 1
        x = np.zeros((6,) + phi.shape[1:])
        for i in range(3):
            for j in range(i, 3):
                ij = _VO[i][j]
                acc = np.zeros(phi.shape[1:])
                for k in range(3):
                    for l in range(3):
                        kl = _VO[k][l]
                        acc = acc + cfac * Cp[..., ij, kl] * (gu[k, l] + em[kl])
                        for v in range(V):
                            acc = acc + Cv[..., ij, kl] * Pphi[v] * tr[v, kl]
                x[ij] = acc
        xh = [ftr(x[m]) for m in range(6)]
        R = [xh[0] * kf[0] + xh[5] * kf[1] + xh[4] * kf[2],
             xh[5] * kf[0] + xh[1] * kf[1] + xh[3] * kf[2],
             xh[4] * kf[0] + xh[3] * kf[1] + xh[2] * kf[2]]
        uh = solve_u(R)
        u = np.array([itr(uh[i]) for i in range(3)])
        gu = np.array([[itr(kf[l] * uh[k]) for l in range(3)] for k in range(3)])
        err = []
        for i in range(3):
            err += [np.sum((u[i] - u_old[i]) ** 2), np.sum(u_old[i] ** 2)]
        ratio = [err[2 * i] / err[2 * i + 1] for i in range(3)]
        if all(r < 1e-7 for r in ratio):
            converged = True
        if niter > 1 and not converged:
            if any(ratio[i] > err_old[2 * i] / err_old[2 * i + 1] for i in range(3)):
                cfac *= newfac
                newfac *= 0.5
                assert newfac >= 1e-7, "newfac is too small"
                niter, converged = 0, False
                continue
        err_old = err
        if niter == 10:
            converged = True
        if not converged or niter < 4:
            continue
        if cfac < 1 - 1e-6:
            cfac = min(cfac + 0.1, 1.0)
            niter, converged = 0, False
            continue
        break
    # elener
    te = sum(Pphi[v][None] * tr[v][:, None, None, None] for v in range(V))
    eps = np.empty((6,) + phi.shape[1:])
    for m in range(3):
        eps[m] = em[m] + gu[m, m] - te[m]
    eps[3] = 2 * em[3] + gu[2, 1] + gu[1, 2] - 2 * te[3]
    eps[4] = 2 * em[4] + gu[2, 0] + gu[0, 2] - 2 * te[4]
    eps[5] = 2 * em[5] + gu[0, 1] + gu[1, 0] - 2 * te[5]
    Ce = np.zeros(phi.shape[1:] + (6, 6))
    for v in range(V):
        Ce += Pphi[v][..., None, None] * sel[phase[v]]
    Ce += (1 - psum)[..., None, None] * sel[1]
    Ce = np.linalg.inv(Ce)
    sig = np.einsum("...ij,j...->i...", Ce, eps)
    el_mat = 0.5 * np.einsum("i...,ij,j...->...", sig, sel[1], sig)
    el_en = (1 - psum) * el_mat
    el_grad = np.zeros_like(phi)
    transsum = tr.sum(axis=1)
    for v in range(V):
        if transsum[v] > float(np.float32(1e-9)):
            el_ppt = 0.5 * np.einsum("i...,ij,j...->...", sig, sel[phase[v]], sig)
            el_en = el_en + el_ppt * Pphi[v]
            fi = phi[v]
            ppr = 30 * fi ** 2 * (fi ** 2 - 2 * fi + 1)
            gsum = (sig[0] * tr[v, 0] + sig[1] * tr[v, 1] + sig[2] * tr[v, 2]
                    + 2 * (sig[3] * tr[v, 3] + sig[4] * tr[v, 4] + sig[5] * tr[v, 5]))
            el_grad[v] = ppr * (el_mat - el_ppt) - gsum * ppr
    return el_en, el_grad, total


def numpy_kks_step(p, cons, phi, elastic=False):
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
    elen, iters = 0.0, 0
    if elastic:
        Pphi = np.array([phi[v] ** 3 * (6 * phi[v] ** 2 - 15 * phi[v] + 10) for v in range(V)])
        el_en, el_grad, iters = numpy_eldis(p, Pphi, phi, ranges)
        fdiff = fdiff + el_grad
        elen = float(np.sum(el_en))
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
    return c_new, phi_new, {"fint": f_int, "fw": float(np.sum(fw)), "fch": float(np.sum(fch)), "elen": elen,
                            "iters": iters}


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


@pytest.mark.parametrize("nvar", [1, 3])
def test_numpy_mirror_of_a_kks_step_with_elasticity(oracle, nvar):
    # The first elastic step (step == elastep0) with heterogeneous cubic moduli (matrix
    # and precipitate stiffnesses not proportional): the zeroth order, the fixed point
    # with its damping and ramp, elener's energy and driving force, on top of the step
    n = 16
    deck = P.parse_input_txt(CF.kks_input_txt(n, nvar, 5, hetero=True))
    p = P.kks_params(deck)
    assert p.step == p.elastep0 and p.step > p.noise_step
    for k in range(p.numph):
        p.wellph[k] = 1.0e8 * (k + 1)
    rng = np.random.default_rng(11 + nvar)
    cons0, phi0 = P.init_fields(deck)
    phi = np.clip(phi0 + rng.uniform(0.0, 0.3, phi0.shape) * (rng.uniform(size=phi0.shape) > 0.15), 0.0, 1.0)
    cons = cons0 + 0.02 * rng.uniform(-1, 1, cons0.shape)
    c1, f1, en = numpy_kks_step(p, cons, phi, elastic=True)
    o = oracle.OracleSim(p)
    o.set_fields(cons, phi)
    d = o.run(1)
    co, fo, _, _ = o.get_fields()
    assert int(d["el_iters"][0]) == en["iters"]
    assert np.max(np.abs(co - c1)) <= 1e-12 * np.max(np.abs(c1))
    assert np.max(np.abs(fo - f1)) <= 1e-12
    for k in ("fint", "fw", "fch", "elen"):
        assert en[k] != 0.0
        assert abs(d[k][0] - en[k]) <= 1e-12 * abs(en[k]), (k, d[k][0], en[k])


@pytest.mark.parametrize("scale", [0.5, 1.5])
def test_numpy_mirror_of_the_elastic_fixed_point_under_contrast(oracle, scale):
    # a precipitate stiffness 1/scale of the deck's, with its C12 raised by 30% (not
    # proportional to the matrix): the fixed point needs 9 iterations (scale 0.5) or stops
    # at the reference's cap of 10 (scale 1.5, ModElastic.f:462-467)
    deck = P.parse_input_txt(CF.kks_input_txt(16, 1, 5, hetero=True))
    p = P.kks_params(deck)
    for k in range(p.numph):
        p.wellph[k] = 1.0e8 * (k + 1)
    c2 = _mat(p, "cela", 1) / scale
    c2[0, 1] *= 1.3
    c2[1, 0] *= 1.3
    p.set_matrix("cela", 1, c2)
    p.set_matrix("sela", 1, np.linalg.inv(c2))
    rng = np.random.default_rng(5)
    cons0, phi0 = P.init_fields(deck)
    phi = np.clip(phi0 + rng.uniform(0.0, 0.3, phi0.shape) * (rng.uniform(size=phi0.shape) > 0.15), 0.0, 1.0)
    cons = cons0 + 0.02 * rng.uniform(-1, 1, cons0.shape)
    c1, f1, en = numpy_kks_step(p, cons, phi, elastic=True)
    o = oracle.OracleSim(p)
    o.set_fields(cons, phi)
    d = o.run(1)
    co, fo, _, _ = o.get_fields()
    assert int(d["el_iters"][0]) == en["iters"] and en["iters"] > 4
    assert np.max(np.abs(co - c1)) <= 1e-12 * np.max(np.abs(c1))
    assert np.max(np.abs(fo - f1)) <= 1e-12
    assert abs(d["elen"][0] - en["elen"]) <= 1e-12 * abs(en["elen"])
