"""Hand-written adjoint of the fused Landau step (one order parameter).

Loss J = 1/(2 N^3) sum [(eta_T - eta*)^2 + (c_T - c*)^2] after T steps; the
target comes from a forward run at other parameters (kappa 1.2, L 0.8, M 1.1,
eps0 0.012) from the same initial fields.  Gradients with respect to kappa
(kappa_c = kappa_eta), L, M, eps0 and the initial eta field are checked in FP64
against central finite differences with h = 1e-4 (relative agreement 1e-4,
the tolerance asked of the adjoint), between checkpoint spacings (bit for bit),
against the FP64 gradient in FP32, and through a torch.autograd.Function.
"""
import numpy as np
import pytest

from helpers import py_uniform
from meumapps_ss_b200 import _lib
from meumapps_ss_b200 import configs as CF
from meumapps_ss_b200 import params as P
from meumapps_ss_b200.sim import Simulation

N, T, K = 32, 24, 5
FD_H = 1e-4
FD_TOL = 1e-4


def deck(kappa=1.0, L=1.0, M=1.0, eps0=0.01, precision=P.PREC_F64, elastic=P.ELAST_HOMOG, n=N):
    p = CF.landau_params(n, 1, [[eps0, eps0, eps0]], dt=0.01, precision=precision, elastic=elastic,
                         kappa_c=kappa, kappa_eta=kappa, M=M, L=L)
    return p


def fields(n=N):
    # ordering region of the free energy: the loss depends on every parameter
    return py_uniform(n, n, n, 1, -21, 0.8, 0.05, 0.5)


def forward_loss(p, c0, e0, ct, et, steps=T):
    s = Simulation(p)
    s.set_fields(c0, e0)
    s.run(steps, diag=False)
    c, e, _, _ = s.get_fields()
    n3 = p.nx * p.ny * p.nz
    return 0.5 / n3 * (np.sum((e - et) ** 2) + np.sum((c - ct) ** 2))


def target(c0, e0, elastic=P.ELAST_HOMOG, n=N, steps=T):
    s = Simulation(deck(1.2, 0.8, 1.1, 0.012, elastic=elastic, n=n))
    s.set_fields(c0, e0)
    s.run(steps, diag=False)
    c, e, _, _ = s.get_fields()
    return c, e


def adjoint(p, c0, e0, ct, et, every=K, steps=T):
    s = Simulation(p)
    s.set_fields(c0, e0)
    return s.adjoint(steps, every, ct, et)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("elastic", [P.ELAST_HOMOG, P.ELAST_NONE])
def test_adjoint_matches_central_differences_fp64(elastic):
    c0, e0 = fields()
    ct, et = target(c0, e0, elastic)
    base = dict(kappa=1.0, L=1.0, M=1.0, eps0=0.01)
    J, g, ge = adjoint(deck(**base, elastic=elastic), c0, e0, ct, et)
    assert rel(J, forward_loss(deck(**base, elastic=elastic), c0, e0, ct, et)) < 1e-12
    adj = {"kappa": g["beta_eta"] / base["kappa"] + g["kappa_c"], "L": g["L"], "M": g["M"],
           "eps0": g["alpha"] / base["eps0"]}
    if elastic == P.ELAST_NONE:
        assert g["alpha"] == 0.0
        del adj["eps0"]
    for k, v in adj.items():
        up, dn = dict(base), dict(base)
        up[k] += FD_H
        dn[k] -= FD_H
        fd = (forward_loss(deck(**up, elastic=elastic), c0, e0, ct, et) -
              forward_loss(deck(**dn, elastic=elastic), c0, e0, ct, et)) / (2 * FD_H)
        assert rel(v, fd) < FD_TOL, (k, v, fd)
    # initial eta field, along a seeded random direction
    d = np.random.default_rng(5).standard_normal(e0.shape)
    p = deck(**base, elastic=elastic)
    fd = (forward_loss(p, c0, e0 + FD_H * d, ct, et) - forward_loss(p, c0, e0 - FD_H * d, ct, et)) / (2 * FD_H)
    assert rel(float(np.sum(ge * d[0])), fd) < FD_TOL


@pytest.mark.gpu
def test_checkpoint_spacing_does_not_change_the_gradient():
    c0, e0 = fields()
    ct, et = target(c0, e0)
    p = deck()
    ref = adjoint(p, c0, e0, ct, et, every=T)
    for every in (1, 7):
        J, g, ge = adjoint(p, c0, e0, ct, et, every=every)
        assert J == ref[0] and g == ref[1] and np.array_equal(ge, ref[2])


@pytest.mark.gpu
def test_fp32_gradient_against_fp64():
    c0, e0 = fields()
    ct, et = target(c0, e0)
    J64, g64, e64 = adjoint(deck(), c0, e0, ct, et)
    J32, g32, e32 = adjoint(deck(precision=P.PREC_F32), c0, e0, ct, et)
    assert rel(J32, J64) < 1e-5
    for k in g64:
        assert rel(g32[k], g64[k]) < 1e-3, (k, g32[k], g64[k])
    assert np.linalg.norm(e32 - e64) / np.linalg.norm(e64) < 1e-3


@pytest.mark.gpu
def test_adjoint_leaves_the_final_state():
    c0, e0 = fields()
    ct, et = target(c0, e0)
    s = Simulation(deck())
    s.set_fields(c0, e0)
    s.adjoint(T, K, ct, et, want_field=False)
    assert s.step == 1 + T
    r = Simulation(deck())
    r.set_fields(c0, e0)
    r.run(T, diag=False)
    assert np.array_equal(s.get_fields()[1], r.get_fields()[1])


@pytest.mark.gpu
def test_torch_autograd_function():
    torch = pytest.importorskip("torch")
    c0, e0 = fields()
    ct, et = target(c0, e0)

    class LandauLoss(torch.autograd.Function):
        """Loss of T steps as a function of (kappa, L, M, eps0) and eta_0; backward is the C-ABI adjoint."""

        @staticmethod
        def forward(ctx, theta, eta0):
            k, L, M, e = (float(x) for x in theta)
            s = Simulation(deck(k, L, M, e))
            s.set_fields(c0, eta0.detach().cpu().numpy())
            J, g, ge = s.adjoint(T, K, ct, et)
            ctx.save_for_backward(torch.tensor([g["beta_eta"] / k + g["kappa_c"], g["L"], g["M"], g["alpha"] / e],
                                               dtype=torch.float64), torch.from_numpy(ge[None]))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            gth, gfield = ctx.saved_tensors
            return gout * gth, gout * gfield

    theta = torch.tensor([1.0, 1.0, 1.0, 0.01], dtype=torch.float64, requires_grad=True)
    eta0 = torch.from_numpy(e0.copy()).requires_grad_(True)
    loss = LandauLoss.apply(theta, eta0)
    loss.backward()
    fd = []
    for i in range(4):
        up = theta.detach().clone()
        dn = theta.detach().clone()
        up[i] += FD_H
        dn[i] -= FD_H
        fd.append((float(LandauLoss.apply(up, eta0.detach())) - float(LandauLoss.apply(dn, eta0.detach()))) / (2 * FD_H))
    for i in range(4):
        assert rel(float(theta.grad[i]), fd[i]) < FD_TOL, i
    assert eta0.grad.shape == eta0.shape


@pytest.mark.gpu
def test_adjoint_rejects_unsupported_handles():
    c0, e0 = fields()
    # heterogeneous elasticity runs on the generic kernels: no adjoint
    p = CF.landau_params(N, 1, [[0.01, 0.01, 0.01]], elastic=P.ELAST_HETERO, ppt_scale=1.5)
    s = Simulation(p)
    s.set_fields(c0, e0)
    with pytest.raises(_lib.MeuError):
        s.adjoint(4, 2, c0, e0)
    q = deck()
    q.flags = P.FLAG_GENERIC
    s = Simulation(q)
    s.set_fields(c0, e0)
    with pytest.raises(_lib.MeuError):
        s.adjoint(4, 2, c0, e0)


# ---------------------------------------------------------------- V variants
def deck_v(nvar, kappa=1.0, L=1.0, M=1.0, alpha=1.0, precision=P.PREC_F64, n=N):
    eig = [[alpha * x for x in row] for row in CF.tetragonal_variants(0.02, -0.005, nvar)]
    return CF.landau_params(n, nvar, eig, dt=0.01, precision=precision, kappa_c=kappa, kappa_eta=kappa, M=M, L=L,
                            cross_w=0.5)


def loss_v(p, c0, e0, ct, et, steps):
    s = Simulation(p)
    s.set_fields(c0, e0)
    s.run(steps, diag=False)
    c, e, _, _ = s.get_fields()
    return 0.5 / p.nx ** 3 * (np.sum((e - et) ** 2) + np.sum((c - ct) ** 2))


@pytest.mark.gpu
@pytest.mark.parametrize("nvar", [2, 3])
def test_multivariant_adjoint_matches_central_differences(nvar):
    """V order parameters: cross-variant Green operator, the cross term w eta_u^2 eta_v^2 and
    the A_uv eigenstrain couplings in the adjoint.  FP64 against central differences
    (h = 1e-4) in kappa, L, M, the eigenstrain scale and the initial eta fields."""
    steps, every = 12, 5
    c0, e0 = py_uniform(N, N, N, nvar, -31, 0.8, 0.05, 0.5)
    t = Simulation(deck_v(nvar, 1.2, 0.8, 1.1, 1.2))
    t.set_fields(c0, e0)
    t.run(steps, diag=False)
    ct, et, _, _ = t.get_fields()
    s = Simulation(deck_v(nvar))
    s.set_fields(c0, e0)
    J, g, ge = s.adjoint(steps, every, ct, et)
    assert ge.shape == e0.shape
    assert rel(J, loss_v(deck_v(nvar), c0, e0, ct, et, steps)) < 1e-12
    adj = {"kappa": g["beta_eta"] + g["kappa_c"], "L": g["L"], "M": g["M"], "alpha": g["alpha"]}
    for k, v in adj.items():
        up, dn = dict(kappa=1.0, L=1.0, M=1.0, alpha=1.0), dict(kappa=1.0, L=1.0, M=1.0, alpha=1.0)
        up[k] += FD_H
        dn[k] -= FD_H
        fd = (loss_v(deck_v(nvar, **up), c0, e0, ct, et, steps) -
              loss_v(deck_v(nvar, **dn), c0, e0, ct, et, steps)) / (2 * FD_H)
        assert rel(v, fd) < FD_TOL, (k, v, fd)
    d = np.random.default_rng(6).standard_normal(e0.shape)
    p = deck_v(nvar)
    fd = (loss_v(p, c0, e0 + FD_H * d, ct, et, steps) - loss_v(p, c0, e0 - FD_H * d, ct, et, steps)) / (2 * FD_H)
    assert rel(float(np.sum(ge * d)), fd) < FD_TOL
    # checkpoint spacing changes nothing, and FP32 follows FP64
    s = Simulation(deck_v(nvar))
    s.set_fields(c0, e0)
    J1, g1, ge1 = s.adjoint(steps, 1, ct, et)
    assert J1 == J and g1 == g and np.array_equal(ge1, ge)
    s = Simulation(deck_v(nvar, precision=P.PREC_F32))
    s.set_fields(c0, e0)
    J32, g32, ge32 = s.adjoint(steps, every, ct, et)
    for k in g:
        assert rel(g32[k], g[k]) < 1e-3, (k, g32[k], g[k])
    assert np.linalg.norm(ge32 - ge) / np.linalg.norm(ge) < 1e-3


@pytest.mark.gpu
def test_deck4_full_size_central_differences():
    """Deck 4 at its own size: 128^3, one variant, 200 steps, checkpoints every 20, target
    from the FP64 forward at kappa 1.2, L 0.8, M 1.1, eps0 0.012.  FP64 gradients in
    kappa, L, M, eps0 and eta_0 (along a seeded direction) against central differences
    with h = 1e-4, within 1e-4."""
    n, steps = 128, 200
    every = CF.ADJOINT_CHECKPOINT_EVERY
    w = CF.adjoint_config(n, P.PREC_F64, **CF.ADJOINT_TARGET)
    c0, e0 = _lib.init_uniform(n, n, n, 1, w.seed, w.c0, w.c_amp, w.eta_amp)
    t = Simulation(w.params)
    t.set_fields(c0, e0)
    t.run(steps, diag=False)
    ct, et, _, _ = t.get_fields()

    def loss(**kw):
        return forward_loss(CF.adjoint_config(n, P.PREC_F64, **kw).params, c0, e0, ct, et, steps=steps)

    st = dict(CF.ADJOINT_START)
    s = Simulation(CF.adjoint_config(n, P.PREC_F64, **st).params)
    s.set_fields(c0, e0)
    J, g, ge = s.adjoint(steps, every, ct, et)
    assert rel(J, loss(**st)) < 1e-12
    adj = {"kappa": g["beta_eta"] / st["kappa"] + g["kappa_c"], "L": g["L"], "M": g["M"],
           "eps0": g["alpha"] / st["eps0"]}
    for k, v in adj.items():
        up, dn = dict(st), dict(st)
        up[k] += FD_H
        dn[k] -= FD_H
        fd = (loss(**up) - loss(**dn)) / (2 * FD_H)
        assert rel(v, fd) < FD_TOL, (k, v, fd)
    d = np.random.default_rng(8).standard_normal(e0.shape)
    p = CF.adjoint_config(n, P.PREC_F64, **st).params
    fd = (forward_loss(p, c0, e0 + FD_H * d, ct, et, steps=steps) -
          forward_loss(p, c0, e0 - FD_H * d, ct, et, steps=steps)) / (2 * FD_H)
    assert rel(float(np.sum(ge * d[0])), fd) < FD_TOL
