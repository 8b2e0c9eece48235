"""The reference's own test suite (tests/test_solver.py, test_fitting.py, test_joint.py,
test_design.py), run against the GPU path, plus the MRF dictionary and config-scale parity against
the C oracle."""
import numpy as np
import pytest

import bmc_oracle as O

pytestmark = pytest.mark.gpu

B0_T = 2.8936
DW = 3.5


def _params(f=0.005, k=300.0, dw=DW, t2_pool_s=0.01, b0=B0_T):
    from bmc_b200.simulation import SimParams
    s = np.float64
    return SimParams(water_r1=s(1 / 3.0), water_r2=s(1 / 0.6), water_f=s(1.0), cest_k=np.array([k]),
                     cest_f=np.array([f]), cest_dw=np.array([dw]), cest_r1=np.array([1.0]),
                     cest_r2=np.array([1.0 / t2_pool_s]), mt_k=s(0), mt_f=s(0), mt_dw=s(0), mt_r1=s(0), mt_r2=s(1),
                     mt_lineshape=np.int32(0), b0=s(b0), gamma=s(267.5153), b0_inhom=s(0), rel_b1=s(1.0))


def _z(p, ppm, b1_uT=1.0, tsat_s=2.0, b0=B0_T):
    from bmc_b200.simulation import initial_state, simulate_z
    from bmc_b200.sequences import cw_saturation
    return simulate_z(p, cw_saturation(ppm, b1_uT=b1_uT, tsat_s=tsat_s, b0_T=b0), initial_state(p), 4)


PPM = np.linspace(-6.0, 6.0, 121)
I_POS = int(np.argmin(np.abs(PPM - DW)))
I_NEG = PPM.size - 1 - I_POS


# ---- physics invariants (tests/test_solver.py:58-130) ------------------------------------------
def test_physics_invariants(cuda):
    z = _z(_params(), PPM)
    assert 0.95 < z[0] < 1.01
    assert abs(PPM[int(np.argmin(z))]) <= 0.5 and z.min() < z[I_POS]
    z0 = _z(_params(f=0.0), PPM)
    assert np.abs(z0 - z0[::-1]).max() < 2e-3
    assert z[I_POS] < z[I_NEG] and z[I_NEG] - z[I_POS] > 0.05
    p = _params()
    assert _z(p, PPM, b1_uT=2.0).mean() < _z(p, PPM, b1_uT=1.0).mean()
    assert _z(p, PPM, tsat_s=4.0).mean() < _z(p, PPM, tsat_s=1.0).mean()
    zk = _z(_params(k=0.0), PPM)
    assert abs(zk[I_NEG] - zk[I_POS]) < 2e-3


@pytest.mark.parametrize("b0", [1.5, 2.8936, 7.0])
def test_ppm_axis_scales_with_field(cuda, b0):
    ppm = np.linspace(0.5, 6.0, 45)
    zw = _z(_params(b0=b0), ppm, b0=b0)
    zn = _z(_params(f=0.0, b0=b0), ppm, b0=b0)
    assert abs(ppm[int(np.argmax(zn - zw))] - DW) < 0.4


# ---- fit recovery (tests/test_fitting.py:29-87) ------------------------------------------------
LADDER = (0.5, 1.0, 1.5, 2.0)
K_TRUE = np.linspace(30.0, 400.0, 8)


@pytest.fixture(scope="module")
def amide_ladder(cuda):
    from bmc_b200.configs import example_config
    from bmc_b200.simulation import to_sim_params, tile_params, initial_state, simulate_z, SimEvent
    from bmc_b200.sequences import cw_saturation
    from bmc_b200.fitting import Experiment
    p = example_config("amide")
    jp = to_sim_params(p)
    ppm = np.linspace(-6.0, 6.0, 41)
    events = Experiment.stack([Experiment(jp, cw_saturation(ppm, b, 2.0, p.system.b0), None, p.mz_loc)
                               for b in LADDER]).events
    n = K_TRUE.size
    base = tile_params(jp, n)._replace(cest_k=K_TRUE[:, None].copy())
    M0 = np.stack([initial_state(jp) for _ in range(n)])
    Z = simulate_z(base, events, M0, p.mz_loc)
    return p, jp, base, events, M0, Z


def test_fit_batch_recovers_k_and_f(amide_ladder):
    from bmc_b200.fitting import FitSpec, FreeParam, fit_batch
    p, jp, base, events, M0, Z = amide_ladder
    spec = FitSpec([FreeParam("k", "cest_k", 0, scale=100.0, lo=5.0, hi=2000.0, x0=150.0),
                    FreeParam("f", "cest_f", 0, scale=0.001, lo=1e-5, hi=0.01, x0=0.0005)])
    X = fit_batch(base, events, M0, p.mz_loc, spec, Z, n_iter=30, skip_first=False, base_batched=True)
    rel = np.abs(X[:, 0] / K_TRUE - 1.0)
    assert rel.max() < 0.05 and rel[K_TRUE > 100].max() < 0.005
    f_true = p.cest_pools[0].f
    assert np.abs(X[:, 1] / f_true - 1.0).max() < 0.03
    flux = np.abs((X[:, 0] * X[:, 1]) / (K_TRUE * f_true) - 1.0).max()
    assert flux <= rel.max() + 1e-9
    assert (X[:, 0] >= 5.0).all() and (X[:, 0] <= 2000.0).all()


def test_fit_batch_matches_the_oracle_lm_step_for_step(amide_ladder):
    """Same start, same damping schedule, float64 on both sides: the device LM and the oracle LM
    land on the same parameters (0.1% target; held to 1e-5 on a noisy, ill-conditioned slow pool)."""
    from bmc_b200.fitting import FitSpec, FreeParam, fit_batch
    p, jp, base, events, M0, Z = amide_ladder
    spec = FitSpec([FreeParam("k", "cest_k", 0, scale=100.0, lo=5.0, hi=2000.0, x0=150.0),
                    FreeParam("f", "cest_f", 0, scale=0.001, lo=1e-5, hi=0.01, x0=0.0005)])
    rng = np.random.default_rng(1)
    zn = Z[:2] + 0.002 * rng.standard_normal(Z[:2].shape)
    sub = type(base)(*[np.asarray(v)[:2] for v in base])
    X = fit_batch(sub, events, M0[:2], p.mz_loc, spec, zn, n_iter=12, skip_first=False, base_batched=True)
    ev = O.Events(*[np.asarray(a) for a in events])
    for i in range(2):
        op = O.Params(*[np.asarray(v)[i] for v in sub])
        x = O.fit_voxel(op, ev, M0[i], [O.Slot("cest_k", 0, 100.0), O.Slot("cest_f", 0, 0.001)], zn[i],
                        [150.0, 0.0005], [5.0, 1e-5], [2000.0, 0.01], n_iter=12)
        np.testing.assert_allclose(X[i], x, rtol=1e-5)     # target 1e-3; rounding differs (Taylor vs Pade)


# ---- joint fits (tests/test_joint.py) -----------------------------------------------------------
K = dict(name="k", field="cest_k", index=0, scale=100.0, lo=5.0, hi=2000.0, x0=150.0)
F = dict(name="f", field="cest_f", index=0, scale=0.001, lo=1e-5, hi=0.01, x0=0.0005)
K_RTOL = 5e-2


@pytest.fixture(scope="module")
def joint3(cuda):
    from bmc_b200.configs import example_config
    from bmc_b200.simulation import to_sim_params, tile_params, initial_state, simulate_z
    from bmc_b200.sequences import cw_saturation
    from bmc_b200.fitting import Experiment
    p = example_config("amide")
    jp = to_sim_params(p)
    ppm = np.linspace(-6.0, 6.0, 41)
    events = Experiment.stack([Experiment(jp, cw_saturation(ppm, b, 2.0, p.system.b0), None, p.mz_loc)
                               for b in LADDER]).events
    true = tile_params(jp, 3)._replace(cest_k=np.array([[40.0], [120.0], [300.0]]))
    m0 = np.stack([initial_state(jp) for _ in range(3)])
    z = simulate_z(true, events, m0, p.mz_loc)
    return p, jp, true, events, m0, z, ppm


def test_plain_spec_joint_equals_fit(joint3):
    from bmc_b200.fitting import Experiment, FitSpec, FreeParam, fit, fit_joint
    p, jp, true, events, m0, z, ppm = joint3
    exp = Experiment(true, events, m0, p.mz_loc)
    spec = FitSpec([FreeParam(**K), FreeParam(**F)])
    a, b = fit(exp, spec, z, n_iter=20), fit_joint(exp, spec, z, n_iter=20)
    np.testing.assert_allclose(b.x, a.x, rtol=1e-9)
    np.testing.assert_allclose(b.z_fit, a.z_fit, rtol=0, atol=1e-10)
    assert b.free.all() and np.isfinite(b.sd).all()


def test_shared_value_is_recovered(joint3):
    from bmc_b200.fitting import Experiment, FitSpec, FreeParam, fit_joint
    p, jp, true, events, m0, z, ppm = joint3
    R2W = FreeParam("r2w", "water_r2", None, scale=10.0, lo=1.0, hi=100.0, x0=14.0, scope="shared")
    start = true._replace(water_r2=np.full(3, 14.0))
    res = fit_joint(Experiment(start, events, m0, p.mz_loc), FitSpec([FreeParam(**K), FreeParam(**F), R2W]), z,
                    n_iter=30)
    assert np.all(res["r2w"] == res["r2w"][0])
    assert res["r2w"][0] == pytest.approx(20.0, rel=5e-3)
    np.testing.assert_allclose(res["k"], [40.0, 120.0, 300.0], rtol=K_RTOL)
    assert np.isfinite(res.sd).all() and res.cost[-1] < res.cost[0] and res.nan_steps == 0


def test_joint_jacobian_is_the_derivative(joint3):
    """fit_joint's assembled Jacobian against central differences of its own residual
    (tests/test_joint.py:347-375), for a shared, a factor, an m_start and a per-block value."""
    from bmc_b200.fitting import Experiment, FitSpec, FreeParam, fit_joint
    p, jp, true, events, m0, z, ppm = joint3
    cases = [
        [FreeParam(**K), FreeParam(**F), FreeParam("r2w", "water_r2", None, 10.0, 1.0, 100.0, 14.0, scope="shared")],
        [FreeParam(**K), FreeParam(**F), FreeParam("r2f", "water_r2", None, 1.0, 0.5, 1.5, 1.0, scope="shared",
                                                   mode="factor"),
         FreeParam("m0", "m_start", None, 1.0, 0.1, 1.0, 0.9, scope="shared")],
        [FreeParam(**K), FreeParam(**F), FreeParam("db0", "b0_inhom", None, 0.01, -0.1, 0.1, 0.0, scope="block",
                                                   mode="add")],
    ]
    for slots in cases:
        d = fit_joint(Experiment(true, events, m0, p.mz_loc), FitSpec(slots), z, n_per_block=ppm.size,
                      _internals=True)
        x = d["x0"] + 0.02 * np.linspace(-1.0, 1.0, d["x0"].size)
        J = d["jac"](x)
        Ja = np.empty_like(J)
        for j in range(x.size):                    # Richardson-extrapolated central differences
            h = 1e-4 * max(1.0, abs(x[j]))
            e = np.zeros(x.size); e[j] = h
            d1 = (d["resid"](x + e) - d["resid"](x - e)) / (2 * h)
            d2 = (d["resid"](x + e / 2) - d["resid"](x - e / 2)) / h
            Ja[:, j] = (4 * d2 - d1) / 3
        rel = np.linalg.norm(J - Ja, axis=0) / np.maximum(np.linalg.norm(Ja, axis=0), 1e-30)
        assert rel.max() < 1e-4, f"{[s.name for s in slots]}: {rel}"      # the reference's own bound


def test_block_offset_and_spread_fits(joint3):
    from bmc_b200.fitting import Experiment, FitSpec, FreeParam, fit_joint
    from bmc_b200.simulation import simulate_z, B0Spread, simulate_spectrum_spread, SimParams
    p, jp, true, events, m0, z, ppm = joint3
    own = np.array([0.0, 0.01, -0.01])
    drift = [0.0, 0.03, -0.02, 0.01]
    n_per = ppm.size
    blocks = []
    for b, dft in enumerate(drift):
        ev = type(events)(*[np.asarray(a)[b * n_per:(b + 1) * n_per] for a in events])
        blocks.append(simulate_z(true._replace(b0_inhom=own + dft), ev, m0, p.mz_loc))
    z2 = np.concatenate(blocks, axis=1)
    DB0 = FreeParam("db0", "b0_inhom", None, scale=0.01, lo=-0.1, hi=0.1, x0=0.0, scope="block", mode="add")
    res = fit_joint(Experiment(true._replace(b0_inhom=own), events, m0, p.mz_loc),
                    FitSpec([FreeParam(**K), FreeParam(**F), DB0]), z2, n_iter=40, n_per_block=n_per)
    np.testing.assert_allclose(res["db0"], drift, atol=2e-3)
    np.testing.assert_allclose(res["k"], [40.0, 120.0, 300.0], rtol=K_RTOL)
    sp = B0Spread(nodes=5)
    one = lambda i: SimParams(*[np.asarray(v)[i] for v in true])
    z3 = np.stack([simulate_spectrum_spread(one(i), events, m0[i], 25.0, sp)[:, p.mz_loc] for i in range(3)])
    SIG = FreeParam("sig", "b0_spread", None, scale=10.0, lo=0.0, hi=60.0, x0=10.0, scope="shared")
    res = fit_joint(Experiment(true, events, m0, p.mz_loc), FitSpec([FreeParam(**K), FreeParam(**F), SIG]), z3,
                    n_iter=30, spread=sp)
    assert res["sig"][0] == pytest.approx(25.0, rel=2e-2)
    np.testing.assert_allclose(res["k"], [40.0, 120.0, 300.0], rtol=K_RTOL)


# ---- CRLB (tests/test_design.py:42-63) -----------------------------------------------------------
def test_crlb_identities(cuda):
    from bmc_b200.configs import example_config
    from bmc_b200.simulation import to_sim_params, initial_state, SimEvent, tile_params
    from bmc_b200.sequences import cw_saturation
    from bmc_b200.fitting import Experiment, FitSpec, FreeParam
    from bmc_b200.design import crlb
    p = example_config("amide")
    jp = to_sim_params(p)
    ppm = np.linspace(-6.0, 6.0, 31)
    rungs = [cw_saturation(ppm, 1.0, 2.0, p.system.b0) for _ in range(3)]
    ev = SimEvent(*[np.concatenate([np.asarray(getattr(e, f)) * (b if f == "rf_amp" else 1)
                                    for e, b in zip(rungs, (0.5, 1.0, 2.0))]) for f in SimEvent._fields])
    exp = Experiment(jp, ev, initial_state(jp), p.mz_loc)
    Kp = FreeParam("k", "cest_k", 0, scale=100.0, lo=5.0, hi=5000.0, x0=150.0)
    Fp = FreeParam("f", "cest_f", 0, scale=0.001, lo=1e-6, hi=0.05, x0=0.0009)
    a, b = crlb(exp, FitSpec([Kp, Fp]), 0.002), crlb(exp, FitSpec([Kp, Fp]), 0.004)
    np.testing.assert_allclose(b.sd, 2 * a.sd, rtol=1e-12)
    twice = Experiment.stack([exp, exp])
    c = crlb(twice, FitSpec([Kp, Fp]), 0.002)
    np.testing.assert_allclose(c.sd, a.sd / np.sqrt(2.0), rtol=1e-9)
    # the bound of k alone is 1/sqrt(F_kk) of the joint Fisher matrix at the same point (the reference
    # compares at two different f and absorbs the difference in a 5e-3 tolerance)
    at_same_f = Experiment(jp._replace(cest_f=np.array([0.0009])), ev, initial_state(jp), p.mz_loc)
    alone = crlb(at_same_f, FitSpec([Kp]), 0.002)
    assert alone.sd[0] == pytest.approx(1.0 / np.sqrt(a.fisher[0, 0]), rel=1e-9)
    assert alone.sd[0] < a.sd[0]
    with pytest.raises(ValueError, match="one sample"):
        crlb(Experiment(tile_params(jp, 2), ev, exp.m0, p.mz_loc), FitSpec([Kp, Fp]), 0.002)


# ---- MRF dictionary and config-scale parity against the C oracle --------------------------------
def test_dictionary_matches_the_oracle(cuda):
    from bmc_b200.configs import example_config
    from bmc_b200.simulation import to_sim_params, initial_state, pack_params
    from bmc_b200.sequences import cw_saturation
    from bmc_b200.mrf import build_param_grid, generate_dictionary
    p = example_config("amide")
    jp = to_sim_params(p)
    ev = cw_saturation(np.linspace(-4, 4, 9), 1.0, 1.0, p.system.b0)
    grid = {"water_r1": [0.5, 0.8, 1.2], "rel_b1": np.linspace(0.7, 1.3, 4), "b0_inhom": [-0.1, 0.0, 0.1]}
    entries, fp = generate_dictionary(jp, ev, initial_state(jp), grid, p.mz_loc, chunk_size=7)
    assert fp.shape == (36, 9) and entries["rel_b1"].shape == (36,)
    pb = build_param_grid(jp, grid)
    want = O.c_simulate_z(pack_params(pb, 36), O.Events(*[np.asarray(a) for a in ev]), initial_state(jp), 1,
                          p.mz_loc)
    np.testing.assert_allclose(fp, want, rtol=0, atol=1e-6)       # fingerprints are float32, like the reference
    with pytest.raises(ValueError, match="Cannot sweep"):
        build_param_grid(to_sim_params(example_config("amide_noe")), {"cest_k": [1.0, 2.0]})


def test_config2_scale_subset_against_the_c_oracle(cuda):
    """The benchmark workload (4 CEST pools + super-Lorentzian MT, 20 Gaussian pulses, 4,023 events),
    a 64-voxel subset: every voxel at 6 offsets against the float64 C oracle (target 1e-5)."""
    import bench
    from bmc_b200.simulation import DeviceEvents, problem
    from bmc_b200 import _lib
    import torch
    import ctypes as C
    P, M0 = bench.voxel_params(64, 4, seed=3)
    ev = bench.pulse_train(101)
    rows = [0, 20, 45, 50, 70, 100]
    ev6 = tuple(np.ascontiguousarray(a[rows]) for a in ev)
    dev_ev = DeviceEvents(O.Events(*ev6))
    z = torch.empty((64, 6), dtype=torch.float64, device="cuda")
    pr = problem(64, 6, ev6[0].shape[1], 4, 10, _lib.F64)
    dP = torch.as_tensor(P).cuda()
    dM = torch.as_tensor(M0).cuda()
    _lib.check(_lib.lib().bmc_simulate(pr, C.c_void_p(dP.data_ptr()), dev_ev.struct, C.c_void_p(dM.data_ptr()),
                                       None, C.c_void_p(z.data_ptr()), _lib.stream_handle()))
    want = O.c_simulate_z(P, O.Events(*ev6), M0, 4, 10)
    err = np.abs(z.cpu().numpy() - want).max()
    print(f"config-2 subset: max |dZ| = {err:.2e}")
    assert err < 1e-9


def test_merged_block_evaluation_equals_the_per_block_launches(joint3):
    """A fit with a per-block value runs every (sample, block) pair in one launch; its Z and Jacobian
    equal those of one launch per block, with a B0 spread, a spread width and m_start among the slots."""
    from bmc_b200.fitting import Experiment, FitSpec, FreeParam, fit_joint
    from bmc_b200.simulation import B0Spread
    p, jp, true, events, m0, z, ppm = joint3
    slots = [FreeParam(**K), FreeParam(**F),
             FreeParam("b1", "rel_b1", None, 1.0, 0.7, 1.3, 1.0, scope="block", mode="factor"),
             FreeParam("sig", "b0_spread", None, 10.0, 0.0, 60.0, 10.0, scope="shared"),
             FreeParam("m0", "m_start", None, 1.0, 0.1, 1.0, 0.9, scope="shared")]
    d = fit_joint(Experiment(true, events, m0, p.mz_loc), FitSpec(slots), z, n_per_block=ppm.size,
                  spread=B0Spread(nodes=5), _internals=True)
    model = d["model"]
    assert model.merged is not None
    loc = d["locs"](d["x0"] + 0.01 * np.linspace(-1.0, 1.0, d["x0"].size))
    Zm, Jm = model.evaluate(loc)
    model.merged = None
    Zb, Jb = model.evaluate(loc)
    np.testing.assert_allclose(Zm, Zb, rtol=0, atol=1e-13)
    np.testing.assert_allclose(Jm, Jb, rtol=1e-12, atol=1e-14)
