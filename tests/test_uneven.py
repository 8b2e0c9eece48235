"""Uneven batches on the GPU: voxels of different pool counts, offsets and pulse trains in one batch.

Each voxel must get what its own shape class gives (the reference runs one class per call), the
float64 oracle's Z, and the joint fit with a value shared by every voxel must follow the oracle's dense
joint LM (fitting/joint.py:149-162) step for step. Tolerances: 1e-13 against the uniform path (same
kernels), 1e-10 in Z against the oracle, 1e-6 relative in the fitted values against the oracle LM.
"""
import numpy as np
import pytest

import bmc_oracle as O

pytestmark = pytest.mark.gpu

GAMMA = 267.5153
POOLS = [(3.5, 1.0, 0.1), (2.0, 1.0, 0.1), (1.0, 1.0, 0.1)]


def pulse_table(ppm, b1s, n_pulses, tp=0.05, gap=0.005, b0=3.0):
    """Rows = every (B1, offset); each row n_pulses x (block pulse tp, gap), then the readout."""
    from bmc_b200.simulation import SimEvent
    rows = [(b, p) for b in b1s for p in ppm]
    n = len(rows)
    ne = 2 * n_pulses + 1
    typ = np.tile(np.int32([1, 0] * n_pulses + [3]), (n, 1))
    dt = np.tile([tp, gap] * n_pulses + [0.0], (n, 1))
    amp = np.array([[b * GAMMA / (2 * np.pi), 0.0] * n_pulses + [0.0] for b, _ in rows])
    fr = np.array([[p * 42.5764 * b0, 0.0] * n_pulses + [0.0] for _, p in rows])
    adc = np.tile(np.int32([-1] * (ne - 1) + [0]), (n, 1))
    return SimEvent(typ, dt, amp, np.zeros((n, ne)), fr, adc)


def voxel(nc, rng, table):
    from bmc_b200.fitting import Experiment
    from bmc_b200.simulation import SimParams, initial_state
    pools = POOLS[:nc]
    p = SimParams(water_r1=np.float64(1 / 1.3), water_r2=np.float64(1 / rng.uniform(0.04, 0.1)),
                  water_f=np.float64(1.0), cest_k=rng.uniform(50, 2000, nc), cest_f=rng.uniform(5e-4, 5e-3, nc),
                  cest_dw=np.array([q[0] for q in pools]), cest_r1=np.array([1 / q[1] for q in pools]),
                  cest_r2=np.array([1 / q[2] for q in pools]), mt_k=np.float64(0.0), mt_f=np.float64(0.0),
                  mt_dw=np.float64(0.0), mt_r1=np.float64(0.0), mt_r2=np.float64(1.0), mt_lineshape=np.int64(0),
                  b0=np.float64(3.0), gamma=np.float64(GAMMA), b0_inhom=np.float64(rng.uniform(-0.1, 0.1)),
                  rel_b1=np.float64(1.0))
    return Experiment(p, table, initial_state(p), 2 * (1 + nc))


@pytest.fixture(scope="module")
def mixed(cuda):
    rng = np.random.default_rng(5)
    tables = [pulse_table(np.linspace(-4, 4, 5), (1.0, 2.0), 1), pulse_table(np.linspace(-5, 5, 3), (0.5, 1.5), 3),
              pulse_table(np.array([-3.5, 0.0, 2.0, 3.5]), (1.0,), 2)]
    exps = [voxel(1 + (i % 3), rng, tables[(i * 7) % 3]) for i in range(18)]
    return exps


def test_each_voxel_gets_its_own_class_result(mixed):
    from bmc_b200.simulation import simulate_z
    from bmc_b200.uneven import UnevenBatch
    zs = UnevenBatch(mixed).simulate()
    for e, z in zip(mixed, zs):
        want = simulate_z(e.params, e.events, e.m0, e.mz_loc)
        np.testing.assert_allclose(z, want, rtol=0, atol=1e-13)


def test_uneven_z_matches_the_oracle(mixed):
    from bmc_b200.uneven import UnevenBatch
    zs = UnevenBatch(mixed).simulate()
    for e, z in list(zip(mixed, zs))[:6]:
        op = O.Params(*[np.asarray(getattr(e.params, f)) for f in O.FIELDS])
        want = O.simulate_spectrum(op, O.Events(*e.events), np.asarray(e.m0))[:, e.mz_loc]
        np.testing.assert_allclose(z, want, rtol=0, atol=1e-10)


def _spec():
    from bmc_b200.fitting import FitSpec, FreeParam
    return FitSpec([FreeParam("k", "cest_k", 0, 100.0, 5.0, 5000.0, 300.0),
                    FreeParam("f", "cest_f", 0, 1e-3, 1e-5, 0.05, 1e-3),
                    FreeParam("k2", "cest_k", 1, 100.0, 5.0, 5000.0, 300.0),
                    FreeParam("r2w", "water_r2", None, 10.0, 5.0, 50.0, 14.0),
                    FreeParam("r1w", "water_r1", None, 1.0, 0.2, 2.0, 0.9, scope="shared")])


def test_joint_fit_follows_the_dense_oracle_lm(mixed):
    """Six voxels (one and two pools, two tables), k, f of pool 1, k of pool 2 where it exists, water R2
    per voxel, water R1 shared: the same iterates as the oracle's dense joint LM."""
    from bmc_b200.simulation import simulate_z
    from bmc_b200.uneven import UnevenBatch, fit_joint_uneven
    exps = [e for e in mixed if len(np.atleast_1d(e.params.cest_k)) <= 2][:6]
    spec = _spec()
    z = [simulate_z(e.params, e.events, e.m0, e.mz_loc) + 0.002 * np.sin(np.arange(np.shape(e.events.dt)[0]))
         for e in exps]
    res = fit_joint_uneven(UnevenBatch(exps), spec, z, n_iter=6)

    # the oracle: one dense problem over [per-voxel k, f, k2, r2w] + [r1w], scaled units
    n, PL = len(exps), 4
    scl = spec.scales
    free = np.ones(n * PL + 1)
    slots = [O.Slot("cest_k", 0), O.Slot("cest_f", 0), O.Slot("cest_k", 1), O.Slot("water_r2", None)]
    for i, e in enumerate(exps):
        if len(np.atleast_1d(e.params.cest_k)) < 2:
            free[i * PL + 2] = 0.0
    x0 = np.concatenate([np.tile(spec.x0_phys[:PL] / scl[:PL], n), [spec.x0_phys[4] / scl[4]]])
    lo = np.concatenate([np.tile(spec.lo_phys[:PL] / scl[:PL], n), [spec.lo_phys[4] / scl[4]]])
    hi = np.concatenate([np.tile(spec.hi_phys[:PL] / scl[:PL], n), [spec.hi_phys[4] / scl[4]]])

    def resid_jac(x, need_jac=True):
        rs, Js = [], []
        for i, e in enumerate(exps):
            nc = len(np.atleast_1d(e.params.cest_k))
            use = [j for j in range(PL) if free[i * PL + j]]
            sl = [slots[j] for j in use] + [O.Slot("water_r1", None)]
            vals = [x[i * PL + j] * scl[j] for j in use] + [x[-1] * scl[4]]
            op = O.write_params(O.Params(*[np.asarray(getattr(e.params, f), np.float64) for f in O.FIELDS]), vals, sl)
            if need_jac:
                Z, J = O.spectrum_jacobian(op, O.Events(*e.events), np.asarray(e.m0), sl, e.mz_loc)
            else:
                Z = O.simulate_spectrum(op, O.Events(*e.events), np.asarray(e.m0))[:, e.mz_loc]
                J = np.zeros((Z.size, len(sl)))
            Jf = np.zeros((Z.size, n * PL + 1))
            for k, j in enumerate(use):
                Jf[:, i * PL + j] = J[:, k] * scl[j]
            Jf[:, -1] = J[:, -1] * scl[4]
            rs.append(Z - z[i])
            Js.append(Jf)
            del nc
        return np.concatenate(rs), np.concatenate(Js)

    xo = O.levenberg_marquardt(resid_jac, x0, lo, hi, n_iter=6, free=free)
    want = xo[:-1].reshape(n, PL) * scl[:PL]
    got = res.x
    mask = free[:-1].reshape(n, PL) > 0
    np.testing.assert_allclose(got[mask], want[mask], rtol=1e-6)
    assert np.isnan(got[~mask]).all()
    assert res.shared == pytest.approx(xo[-1] * scl[4], rel=1e-6)


def test_joint_fit_from_a_cuda_graph_equals_the_eager_loop(mixed):
    """One iteration captured in a CUDA graph and replayed gives the eager loop's iterates bit for bit."""
    from bmc_b200.simulation import simulate_z
    from bmc_b200.uneven import UnevenBatch, fit_joint_uneven
    exps = mixed[:9]
    z = [simulate_z(e.params, e.events, e.m0, e.mz_loc) + 0.001 * np.cos(np.arange(np.shape(e.events.dt)[0]))
         for e in exps]
    a = fit_joint_uneven(UnevenBatch(exps), _spec(), z, n_iter=7, graph=True)
    b = fit_joint_uneven(UnevenBatch(exps), _spec(), z, n_iter=7, graph=False)
    np.testing.assert_array_equal(a.x, b.x)
    np.testing.assert_array_equal(a.cost, b.cost)
    assert a.shared == b.shared


def test_dense_switch_changes_the_path_not_the_result(mixed, tmp_path):
    """The dense-path threshold of a plan (bmc_uneven_set_dense_switch) picks how an event is
    exponentiated, not what comes out (both paths meet the tolerance); the autotuner's choices survive a
    round trip through its JSON file."""
    from bmc_b200 import _lib
    from bmc_b200.autotune import apply_tuning, tune_dense_switch
    from bmc_b200.uneven import UnevenBatch
    batch = UnevenBatch(mixed)
    ref = batch.simulate()
    for norm in (8.0, 1e5):
        for g in batch.groups:
            _lib.check(_lib.lib().bmc_uneven_set_dense_switch(g.plan.plan, norm))
        for a, b in zip(batch.simulate(), ref):
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-12)
    with pytest.raises(RuntimeError, match="dense-path norm"):
        _lib.check(_lib.lib().bmc_uneven_set_dense_switch(batch.groups[0].plan.plan, -1.0))
    path = tmp_path / "tuning.json"
    from bmc_b200 import settings
    from bmc_b200.autotune import plan_key, uses_block_kernel
    settings.use_tangents("forward")              # every plan on the chain kernel: a threshold to tune
    try:
        chosen = tune_dense_switch(batch, candidates=(25.0, 100.0), repeats=1, path=str(path))
        again = apply_tuning(UnevenBatch(mixed), str(path))
    finally:
        settings.use_tangents("auto")
    assert len(chosen) == len(batch.groups) and all(v["dense_switch"] in (25.0, 100.0) for v in chosen.values())
    assert again == {k: v["dense_switch"] for k, v in chosen.items()}
    # automatic mode: the plans on the block kernel have no threshold and are not timed
    auto = tune_dense_switch(batch, candidates=(25.0,), repeats=1)
    for g in batch.groups:
        assert (auto[plan_key(g)]["dense_switch"] is None) == uses_block_kernel(g)


def test_joint_fit_recovers_the_truth(mixed):
    from bmc_b200.simulation import simulate_z
    from bmc_b200.uneven import UnevenBatch, fit_joint_uneven
    spec = _spec()
    z = [simulate_z(e.params, e.events, e.m0, e.mz_loc) for e in mixed]
    res = fit_joint_uneven(UnevenBatch(mixed), spec, z, n_iter=40)
    truth_k = np.array([np.atleast_1d(e.params.cest_k)[0] for e in mixed])
    truth_r2 = np.array([float(e.params.water_r2) for e in mixed])
    assert res.shared == pytest.approx(1 / 1.3, rel=1e-4)
    assert np.median(np.abs(res["k"] / truth_k - 1)) < 1e-3
    assert np.median(np.abs(res["r2w"] / truth_r2 - 1)) < 1e-4
    assert res.cost[-1] < 1e-3 * res.cost[0]


def test_schur_step_in_one_call_and_in_shards_is_the_dense_step(cuda):
    """bmc_schur_step, and bmc_schur_eliminate on two shards + summed sums + bmc_schur_back, against the
    dense damped step of the whole problem (fitting/joint.py:149-162)."""
    torch = cuda
    from bmc_b200 import _lib
    rng = np.random.default_rng(11)
    n, PL, lam = 37, 4, 0.03
    P = PL + 1
    H = np.stack([(lambda J: J.T @ J)(rng.normal(size=(20, P))) for _ in range(n)])
    g = rng.normal(size=(n, P))
    free = np.ones((n, PL))
    free[::4, 2] = 0.0
    d_want, ds_want = O.joint_step_dense(H, g, free, lam, 1)
    L = _lib.lib()
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64)).cuda()
    dH, dg, dfree = dev(H), dev(g), dev(free)
    d = torch.empty((n, PL), dtype=torch.float64, device="cuda")
    ds = torch.empty(1, dtype=torch.float64, device="cuda")
    work = torch.empty((2 * PL + 4) * n + 4, dtype=torch.float64, device="cuda")
    _lib.check(L.bmc_schur_step(n, PL, 1, _lib.ptr(dH), _lib.ptr(dg), _lib.ptr(dfree), lam, None, _lib.ptr(d),
                                _lib.ptr(ds), _lib.ptr(work), _lib.stream_handle()))
    np.testing.assert_allclose(d.cpu().numpy(), d_want, rtol=1e-10, atol=1e-12)
    assert float(ds.item()) == pytest.approx(ds_want, rel=1e-10)
    # two shards, the damping read from device memory
    d_lam = torch.tensor([lam], dtype=torch.float64, device="cuda")
    cut = 15
    parts = [(slice(0, cut), cut), (slice(cut, n), n - cut)]
    works = [torch.empty((2 * PL + 4) * m, dtype=torch.float64, device="cuda") for _, m in parts]
    sums = [torch.empty(4, dtype=torch.float64, device="cuda") for _ in parts]
    for (sl, m), wk, sm in zip(parts, works, sums):
        _lib.check(L.bmc_schur_eliminate(m, PL, 1, _lib.ptr(dH[sl].contiguous()), _lib.ptr(dg[sl].contiguous()),
                                         _lib.ptr(dfree[sl].contiguous()), -1.0, _lib.ptr(d_lam), _lib.ptr(wk),
                                         _lib.ptr(sm), _lib.stream_handle()))
    total = sums[0] + sums[1]
    for (sl, m), wk in zip(parts, works):
        dd = torch.empty((m, PL), dtype=torch.float64, device="cuda")
        _lib.check(L.bmc_schur_back(m, PL, 1, _lib.ptr(total), -1.0, _lib.ptr(d_lam), _lib.ptr(wk), _lib.ptr(dd),
                                    _lib.ptr(ds), _lib.stream_handle()))
        np.testing.assert_allclose(dd.cpu().numpy(), d_want[sl], rtol=1e-10, atol=1e-12)
    assert float(ds.item()) == pytest.approx(ds_want, rel=1e-10)
