"""optimize_design (design/optimize.py:43-113): the reference's own test on the GPU, and the cost and its
gradient against the float64 oracle (oracle Jacobians through scipy's expm_frechet). The gradient is exact
from the simulation on (bmc_simulate_design_jvp); the oracle differentiates its exact Jacobian in d by a
five-point stencil. Tolerances: cost 1e-8 relative; dJ/dd 2e-7 of its largest entry; the gradient 1e-7
(amplitude ladder) and 1e-6 (every kind of input); central differences of the GPU cost 1e-5.
"""
import numpy as np
import pytest

import bmc_oracle as O

PPM = np.linspace(-6.0, 6.0, 31)
SIGMA = 0.002


def _setup():
    from bmc_b200.configs import example_config
    from bmc_b200.fitting import FitSpec, FreeParam
    from bmc_b200.sequences import cw_saturation
    from bmc_b200.simulation import initial_state, to_sim_params
    p = example_config("amide")
    jp = to_sim_params(p)
    rungs = [cw_saturation(PPM, b1_uT=1.0, tsat_s=2.0, b0_T=p.system.b0) for _ in range(3)]
    K = FreeParam("k", "cest_k", 0, scale=100.0, lo=5.0, hi=5000.0, x0=150.0)
    F = FreeParam("f", "cest_f", 0, scale=0.001, lo=1e-6, hi=0.05, x0=0.0009)
    return p, jp, initial_state(jp), rungs, FitSpec([K, F])


def _ladder(setup, b1):
    """The three rungs at the amplitudes b1 (uT): the amplitude scales rf_amp linearly."""
    from bmc_b200.fitting import Experiment
    from bmc_b200.simulation import SimEvent
    p, jp, m0, rungs, _ = setup
    ev = SimEvent(*[np.concatenate(a, axis=0) for a in
                    zip(*[e._replace(rf_amp=np.asarray(e.rf_amp, np.float64) * b) for e, b in zip(rungs, b1)])])
    return Experiment(jp, ev, m0, p.mz_loc)


def test_design_bounds_are_checked():
    from bmc_b200.design import optimize_design
    setup = _setup()
    with pytest.raises(ValueError, match="lo < d0 < hi"):
        optimize_design(lambda d: _ladder(setup, d), setup[4], d0=[0.05, 1.0, 2.0], lo=[0.1] * 3, hi=[3.0] * 3,
                        sigma=SIGMA, truths=[[150.0, 0.0009]], n_steps=1)
    with pytest.raises(ValueError, match="targets"):
        optimize_design(lambda d: _ladder(setup, d), setup[4], d0=[0.5, 1.0, 2.0], lo=[0.1] * 3, hi=[3.0] * 3,
                        sigma=SIGMA, truths=[[150.0, 0.0009]], targets=["t1"], n_steps=1)


@pytest.mark.gpu
def test_optimising_the_amplitudes_lowers_the_bound(cuda):
    from bmc_b200.design import optimize_design
    setup = _setup()
    res = optimize_design(lambda d: _ladder(setup, d), setup[4], d0=[0.5, 1.0, 2.0], lo=[0.1] * 3, hi=[3.0] * 3,
                          sigma=SIGMA, truths=[[150.0, 0.0009]], n_steps=15, lr=0.1)
    assert res.cost[-1] < res.cost[0]
    assert np.all(res.design > 0.1) and np.all(res.design < 3.0)
    assert np.all(res.rel_sd_end <= res.rel_sd_start * 1.0001)


def _oracle_cost(setup, d, truths):
    p, jp, m0, rungs, spec = setup
    ex = _ladder(setup, d)
    op = O.Params(*[np.asarray(getattr(jp, f), np.float64) for f in O.FIELDS])
    slots = [O.Slot("cest_k", 0), O.Slot("cest_f", 0)]
    ev = O.Events(*[np.asarray(a, np.float64) if np.asarray(a).dtype.kind == "f" else np.asarray(a) for a in ex.events])
    total = 0.0
    for x in truths:
        _, J = O.spectrum_jacobian(O.write_params(op, x, slots), ev, np.asarray(m0), slots, p.mz_loc)
        var = np.diag(np.linalg.inv(J.T @ J / SIGMA ** 2))
        total += float(np.sum(var / np.asarray(x) ** 2))
    return total / len(truths)


@pytest.mark.gpu
def test_cost_and_gradient_match_the_oracle(cuda):
    from bmc_b200.design import design_cost
    setup = _setup()
    truths = [[150.0, 0.0009], [60.0, 0.002]]
    d = np.array([0.5, 1.0, 2.0])
    c = design_cost(lambda dd: _ladder(setup, dd), setup[4], d, SIGMA, truths, ("k", "f"))
    assert c == pytest.approx(_oracle_cost(setup, d, truths), rel=1e-8)
    h = 1e-4 * 2.9
    for i in range(3):
        e = np.zeros(3)
        e[i] = h
        g = (design_cost(lambda dd: _ladder(setup, dd), setup[4], d + e, SIGMA, truths, ("k", "f")) -
             design_cost(lambda dd: _ladder(setup, dd), setup[4], d - e, SIGMA, truths, ("k", "f"))) / (2 * h)
        go = (_oracle_cost(setup, d + e, truths) - _oracle_cost(setup, d - e, truths)) / (2 * h)
        assert g == pytest.approx(go, rel=1e-5)


# ------------------------------------------------------------------------------------------------
# the exact design gradient (bmc_simulate_design_jvp): dJ/dd against the oracle's exact Jacobian
# differentiated in d by a five-point stencil (truncation ~1e-12 relative at these steps)
# ------------------------------------------------------------------------------------------------
def _oracle_J(ex, x, slots):
    op = O.Params(*[np.asarray(getattr(ex.params, f), np.float64) for f in O.FIELDS])
    ev = O.Events(*[np.asarray(a, np.float64) if np.asarray(a).dtype.kind == "f" else np.asarray(a) for a in ex.events])
    return O.spectrum_jacobian(O.write_params(op, x, slots), ev, np.asarray(ex.m0, np.float64), slots, ex.mz_loc)[1]


def _oracle_dJ(build, d, truths, slots, steps):
    """(J, dJ, cost, dcost): the oracle's J at d and its stencil derivatives in every setting, with the
    cost of design_cost and the same stencil of it."""
    def cost_of(Js):
        return np.mean([np.sum(np.diag(np.linalg.inv(J.T @ J / SIGMA ** 2)) / np.asarray(x) ** 2)
                        for x, J in zip(truths, Js)])
    J0 = [_oracle_J(build(d), x, slots) for x in truths]
    dJ, dc = [], []
    for i in range(len(d)):
        at = {}
        for k in (-2, -1, 1, 2):
            dd = np.array(d, np.float64, copy=True)
            dd[i] += k * steps[i]
            at[k] = [_oracle_J(build(dd), x, slots) for x in truths]
        st = lambda f: (-f(2) + 8 * f(1) - 8 * f(-1) + f(-2)) / (12 * steps[i])
        dJ.append(np.stack([st(lambda k: at[k][t]) for t in range(len(truths))]))
        dc.append(st(lambda k: cost_of(at[k])))
    return np.stack(J0), np.stack(dJ), cost_of(J0), np.array(dc)


def _rich_setup():
    from bmc_b200.configs import example_config
    from bmc_b200.fitting import FitSpec, FreeParam
    from bmc_b200.sequences import cw_saturation
    from bmc_b200.simulation import initial_state, to_sim_params
    p = example_config("amide_noe_mt")
    jp = to_sim_params(p)
    ppm = np.linspace(-6.0, 6.0, 9)
    rung = cw_saturation(ppm, b1_uT=1.0, tsat_s=1.0, b0_T=p.system.b0)
    K = FreeParam("k", "cest_k", 0, scale=100.0, lo=5.0, hi=5000.0, x0=150.0)
    F = FreeParam("f", "cest_f", 0, scale=0.001, lo=1e-6, hi=0.05, x0=0.0009)
    return p, jp, initial_state(jp), rung, FitSpec([K, F])


def _rich(setup, d):
    """Every input the second-order kernel differentiates moves with d: d[0] scales rung 1's amplitude,
    d[1] is rung 2's saturation time (0.02 s: its rows take the Taylor path; 1 s rungs the dense one),
    d[2] shifts rung 3's offsets (x 50 Hz), d[3] is rung 1's RF phase, d[4] scales the main field b0 (a
    parameter) and d[5] the start state. At b0 x 1.05 no row's MT offset sits where the super-Lorentzian
    switches from its direct form to the Hermite bridge (|delta| = w0, a kink of the lineshape itself:
    at b0 x 1 two rows do, and a central difference across it is not a derivative)."""
    from bmc_b200.fitting import Experiment
    from bmc_b200.simulation import SimEvent
    p, jp, m0, rung, _ = setup
    f = lambda a: np.asarray(a, np.float64)
    r1 = rung._replace(rf_amp=f(rung.rf_amp) * d[0], rf_phase=np.where(f(rung.dt) > 0, d[3], 0.0))
    r2 = rung._replace(dt=np.where(f(rung.dt) > 0, d[1], 0.0))
    r3 = rung._replace(rf_freq=f(rung.rf_freq) + np.where(f(rung.dt) > 0, 50.0 * d[2], 0.0))
    ev = SimEvent(*[np.concatenate(a, axis=0) for a in zip(r1, r2, r3)])
    return Experiment(jp._replace(b0=float(np.asarray(jp.b0)) * d[4]), ev, np.asarray(m0, np.float64) * d[5],
                      p.mz_loc)


@pytest.mark.gpu
def test_design_derivative_matches_the_oracle(cuda):
    """dJ/dd of every kind of input (event amplitude, duration on both paths, frequency, phase, a
    parameter, the start state) on a model with MT (super-Lorentzian), and the cost's exact gradient."""
    from bmc_b200.design import design_cost_and_gradient, design_jacobians, jacobians
    setup = _rich_setup()
    build = lambda d: _rich(setup, d)
    d = np.array([0.8, 0.02, 0.3, 0.4, 1.05, 1.0])
    steps = np.array([1e-3, 2e-5, 1e-3, 1e-3, 1e-3, 1e-3])
    truths = [[150.0, 0.0009], [60.0, 0.002]]
    J, dJ = design_jacobians(build, setup[4], d, truths, steps)
    np.testing.assert_allclose(J, jacobians(build(d), setup[4], truths), rtol=0, atol=1e-10 * np.abs(J).max())
    slots = [O.Slot("cest_k", 0), O.Slot("cest_f", 0)]
    # oracle steps: halving each changes its stencil by < 5e-8 of the largest entry (on resonance, Z's
    # f-derivative bends fast with the amplitude: a step of 2e-3 is off by 3e-3 there)
    Jo, dJo, co, dco = _oracle_dJ(build, d, truths, slots, np.array([5e-4, 1e-5, 5e-4, 5e-4, 5e-4, 5e-4]))
    np.testing.assert_allclose(J, Jo, rtol=0, atol=1e-9 * np.abs(Jo).max())
    for i in range(d.size):
        scale = max(np.abs(dJo[i]).max(), 1e-3 * np.abs(Jo).max())
        np.testing.assert_allclose(dJ[i], dJo[i], rtol=0, atol=2e-7 * scale, err_msg=f"setting {i}")
    c, g = design_cost_and_gradient(build, setup[4], d, SIGMA, truths, ("k", "f"), steps)
    assert c == pytest.approx(co, rel=1e-8)
    np.testing.assert_allclose(g, dco, rtol=1e-6, atol=1e-9 * np.abs(dco).max())


@pytest.mark.gpu
def test_exact_gradient_of_the_amplitude_ladder(cuda):
    """The reference test's design (three CW rungs, amplitudes): the exact gradient against the oracle
    cost's stencil derivative at 1e-7, and the central differences of the GPU cost agree with it."""
    from bmc_b200.design import design_cost, design_cost_and_gradient
    setup = _setup()
    build = lambda dd: _ladder(setup, dd)
    truths = [[150.0, 0.0009], [60.0, 0.002]]
    d = np.array([0.5, 1.0, 2.0])
    c, g = design_cost_and_gradient(build, setup[4], d, SIGMA, truths, ("k", "f"), np.full(3, 2.9e-3))
    slots = [O.Slot("cest_k", 0), O.Slot("cest_f", 0)]
    _, _, co, dco = _oracle_dJ(build, d, truths, slots, np.full(3, 5e-4))
    assert c == pytest.approx(co, rel=1e-8)
    np.testing.assert_allclose(g, dco, rtol=1e-7)
    h = 1e-4 * 2.9
    for i in range(3):
        e = np.zeros(3)
        e[i] = h
        gc = (design_cost(build, setup[4], d + e, SIGMA, truths, ("k", "f")) -
              design_cost(build, setup[4], d - e, SIGMA, truths, ("k", "f"))) / (2 * h)
        assert gc == pytest.approx(g[i], rel=1e-5)


def test_build_direction_is_exact_for_affine_builds_and_checks_the_table():
    """The host side of the exact gradient: the five-point stencil of build(d) gives the table's change per
    unit of a setting exactly (to rounding) for a build affine in it, and refuses a design that changes
    the table's shape or event types as it moves."""
    from bmc_b200.design import _build_direction
    setup = _setup()
    build = lambda dd: _ladder(setup, dd)
    d = np.array([0.5, 1.0, 2.0])
    ev, p_dir, m_dir = _build_direction(build, d, 1, 1e-3, build(d))
    base = np.asarray(setup[3][1].rf_amp, np.float64)
    n = base.shape[0]
    want = np.zeros((3 * n, base.shape[1]))
    want[n:2 * n] = base                                  # rung 2's amplitude moves with d[1], 1:1
    np.testing.assert_allclose(ev[1], want, rtol=0, atol=1e-9 * np.abs(base).max())
    for j in (0, 2, 3):                                   # dt, phase, frequency do not move
        assert np.abs(ev[j]).max() < 1e-9
    assert np.abs(p_dir).max() == 0.0 and np.abs(m_dir).max() == 0.0

    def growing(dd):                                      # a setting that adds events: not differentiable
        ex = build(dd)
        if dd[0] > 0.5:
            from bmc_b200.fitting import Experiment
            from bmc_b200.simulation import SimEvent
            e = ex.events
            ev2 = SimEvent(*[np.concatenate([np.asarray(a), np.asarray(a)[:, :1]], axis=1) for a in e])
            return Experiment(ex.params, ev2, ex.m0, ex.mz_loc)
        return ex
    with pytest.raises(ValueError, match="shape and event types"):
        _build_direction(growing, d, 0, 1e-3, build(d))
