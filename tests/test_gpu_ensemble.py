"""Batched ensemble, schedule variants and graph replay of the fused Landau step.

* An ensemble member's step is the single-handle step: fields and per-step
  diagnostics of every member equal those of its own Simulation bit for bit
  (same kernels, same schedule, same reduction order), in FP32 and FP64, over
  runs long enough to replay the CUDA graph.
* Every instantiated schedule (radix plan, plane threads, column tile) gives the
  FP64 oracle's fields to 1e-10.
* The autotuned ensemble picks instantiated schedules and stays within the FP32
  tolerance of the FP64 path.
* The persistent ensemble (one launch per run of steps, every size's passes as work
  items) gives each member's single-handle fields on its schedule bit for bit.
"""
import numpy as np
import pytest

from helpers import active_landau
from meumapps_ss_b200 import _lib
from meumapps_ss_b200 import configs as CF
from meumapps_ss_b200 import params as P
from meumapps_ss_b200.sim import Ensemble, Simulation, schedule_candidates

TOL = 1e-10


def _members(precision, sizes=(32, 48, 32, 64, 48), nvars=(1, 1, 2, 1, 3)):
    out = []
    for i, (n, nv) in enumerate(zip(sizes, nvars)):
        p, c, e = active_landau(n=n, nvar=nv, precision=precision, seed=-(11 + i))
        p.lan_b = 0.7 + 0.2 * i
        out.append((p, c, e))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [P.PREC_F64, P.PREC_F32])
def test_ensemble_equals_single_handles(precision):
    ms = _members(precision)
    ens = Ensemble([m[0] for m in ms])
    for i, (p, c, e) in enumerate(ms):
        ens.set_fields(i, c, e)
    de = ens.run(21)  # one eager step, two 8-step graph replays, four eager steps
    assert ens.step == ms[0][0].step + 21
    for i, (p, c, e) in enumerate(ms):
        s = Simulation(p)
        s.set_fields(c, e)
        ds = s.run(21)
        cs, es, _, _ = s.get_fields()
        ce, ee, _ = ens.get_fields(i)
        assert np.array_equal(cs, ce), i
        assert np.array_equal(es, ee), i
        for k in ("fint", "fch", "elen", "etot", "cmin", "cmax", "phimax", "solid_now", "cavg"):
            assert np.array_equal(ds[k], de[i][k]), (i, k)
        assert np.array_equal(ds["step"], de[i]["step"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [P.PREC_F32, P.PREC_F64])
def test_persistent_ensemble_equals_single_handles(precision):
    """MEU_ENS_PERSISTENT: after the first (per-bucket) step, every pass of every member
    of five grid sizes runs as work items of one launch per run of up to 64 steps; each
    member's fields equal those of its own handle on the persistent schedule bit for bit."""
    sizes = (32, 48, 64, 32, 96, 128)
    ms = _members(precision, sizes=sizes, nvars=(1,) * len(sizes))
    ens = Ensemble([m[0] for m in ms], persistent=True)
    tm = 16 if precision == P.PREC_F32 else 8
    for i, (p, c, e) in enumerate(ms):
        assert ens.schedule(i)[:3] == (2, 256, tm)
        ens.set_fields(i, c, e)
    n0 = ens.launch_count
    de = ens.run(70)  # one per-bucket step, then persistent launches of 64 and 5 steps
    buckets = len(set(sizes))
    assert ens.launch_count - n0 == 7 * buckets + 2
    assert ens.step == ms[0][0].step + 70
    for i, (p, c, e) in enumerate(ms):
        s = Simulation(p)
        s.set_schedule(2, 256, tm)
        s.set_fields(c, e)
        ds = s.run(70)
        cs, es, _, _ = s.get_fields()
        ce, ee, _ = ens.get_fields(i)
        assert np.array_equal(cs, ce), i
        assert np.array_equal(es, ee), i
        # the energies: same sums, but the elastic energy is a difference of two large
        # quadratic forms, and the compiler fuses multiply-adds differently in the
        # persistent kernel (a separately compiled body), which the cancellation lifts to
        # ~1e-9 relative in FP64
        for k in ("fint", "fch", "elen", "etot", "cmin", "cmax", "phimax", "solid_now", "cavg"):
            assert np.allclose(ds[k], de[i][k], rtol=1e-8, atol=0.0), (i, k)
        assert np.array_equal(ds["step"], de[i]["step"])


@pytest.mark.gpu
def test_persistent_ensemble_rules():
    ms = _members(P.PREC_F32, sizes=(32, 48), nvars=(1, 2))
    with pytest.raises(_lib.MeuError) as ex:
        Ensemble([m[0] for m in ms], persistent=True)
    assert ex.value.code == 103  # MEU_ERR_UNSUPPORTED


@pytest.mark.gpu
def test_ensemble_launches_per_bucket():
    ms = _members(P.PREC_F32)
    ens = Ensemble([m[0] for m in ms])
    for i, (p, c, e) in enumerate(ms):
        ens.set_fields(i, c, e)
    n0 = ens.launch_count
    ens.run(16)
    buckets = len({(p.nx, p.nvar) for p, _, _ in ms})
    # per bucket and step, whatever the member count: five kernels, plus the theta
    # transform on the first step after new fields and, on the ensemble's first step,
    # the one-time condition test of Q(k)
    assert ens.launch_count - n0 == (7 + 15 * 5) * buckets


@pytest.mark.gpu
def test_graph_replay_equals_stepwise():
    p, c, e = active_landau(n=48, nvar=2, precision=P.PREC_F32, seed=-5)
    a = Simulation(p)
    a.set_fields(c, e)
    da = a.run(19)
    b = Simulation(p)
    b.set_fields(c, e)
    db = [b.run(1) for _ in range(19)]
    ca, ea, _, _ = a.get_fields()
    cb, eb, _, _ = b.get_fields()
    assert np.array_equal(ca, cb) and np.array_equal(ea, eb)
    assert np.array_equal(da["etot"], np.concatenate([d["etot"] for d in db]))


@pytest.mark.gpu
@pytest.mark.parametrize("n,nvar", [(32, 2), (48, 1)])
def test_every_schedule_matches_oracle(oracle, n, nvar):
    p, c, e = active_landau(n=n, nvar=nvar)
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    do = o.run(24)
    co, eo, _, _ = o.get_fields()
    cands = schedule_candidates(n, True)
    assert len(cands) >= 6
    for sch in cands:
        g = Simulation(p)
        g.set_schedule(*sch)
        assert g.schedule == sch
        g.set_fields(c, e)
        dg = g.run(24)
        cg, eg, _, _ = g.get_fields()
        assert np.max(np.abs(cg - co)) <= TOL, sch
        assert np.max(np.abs(eg - eo)) <= TOL, sch
        assert np.max(np.abs(dg["etot"] - do["etot"]) / np.abs(do["etot"])) < 1e-9, sch


@pytest.mark.gpu
def test_set_schedule_rules():
    p, c, e = active_landau(n=32, nvar=1)
    g = Simulation(p)
    with pytest.raises(_lib.MeuError):
        g.set_schedule(0, 384, 8)  # no such variant
    g.set_fields(c, e)
    with pytest.raises(_lib.MeuError):
        g.set_schedule(1, 256, 4)  # the spectral-state layout is fixed by then
    q = CF.landau_params(32, 1, [[0.01, 0.01, 0.01]])
    q.flags = P.FLAG_GENERIC
    h = Simulation(q)
    assert h.schedule == (0, 0, 1)  # generic path: radix plan, column-tile factor
    h.set_schedule(2, 0, 2)
    assert h.schedule == (2, 0, 2)
    with pytest.raises(_lib.MeuError):
        h.set_schedule(1, 0, 1)


@pytest.mark.gpu
def test_autotuned_ensemble_fp32_vs_fp64():
    ws = CF.ensemble_config(6, precision=P.PREC_F32, sizes=(32, 48, 64))
    e32 = Ensemble([w.params for w in ws], autotune=True)
    e64 = Ensemble([P.MeuParams.copy(w.params) for w in CF.ensemble_config(6, precision=P.PREC_F64, sizes=(32, 48, 64))])
    for i, w in enumerate(ws):
        sch = e32.schedule(i)
        assert sch[:3] in schedule_candidates(w.params.nx, False)
        c, e = CF.uniform_fields(w)
        e32.set_fields(i, c, e)
        e64.set_fields(i, c, e)
    e32.run(40, diag=False)
    e64.run(40, diag=False)
    for i in range(len(ws)):
        c1, f1, _ = e32.get_fields(i)
        c2, f2, _ = e64.get_fields(i)
        assert np.linalg.norm(c1 - c2) / np.linalg.norm(c2) < 1e-6
        assert np.linalg.norm(f1 - f2) / np.linalg.norm(f2) < 1e-5


@pytest.mark.gpu
def test_single_handle_autotune_flag(oracle):
    p, c, e = active_landau(n=32, nvar=1)
    p.flags = P.FLAG_AUTOTUNE
    g = Simulation(p)
    assert g.schedule in schedule_candidates(32, True)
    g.set_fields(c, e)
    g.run(10)
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    o.run(10)
    cg, eg, _, _ = g.get_fields()
    co, eo, _, _ = o.get_fields()
    assert np.max(np.abs(cg - co)) <= TOL and np.max(np.abs(eg - eo)) <= TOL
