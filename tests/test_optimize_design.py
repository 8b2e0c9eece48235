"""optimize_design (design/optimize.py:43-113): the reference's own test on the GPU, and the cost and its
gradient against the float64 oracle (oracle Jacobians through scipy's expm_frechet, same central
differences). Tolerances: cost 1e-8 relative, gradient 1e-5 relative.
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
