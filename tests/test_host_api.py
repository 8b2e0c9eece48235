"""Host-side API that needs no GPU: parameter and event builders, layouts, validation messages and
the physics-free LM, against the reference's behaviour (golden vectors / its tests' assertions)."""
import numpy as np
import pytest

import bmc_oracle as O
from bmc_b200.configs import example_config
from bmc_b200.fitting import (Experiment, FitSpec, FreeParam, fit, fit_joint, field_row, levenberg_marquardt,
                              write_params)
from bmc_b200.sequences import cw_saturation, hz_per_ppm
from bmc_b200.simulation import (SimEvent, SimParams, initial_state, pack_params, pad_events, to_sim_params,
                                 state_size, B0Spread, tile_params)
from conftest import golden


def test_cw_saturation_stack_and_pad_match_the_reference():
    d = golden("events")
    ev = cw_saturation(np.linspace(-6, 6, 7), 1.5, 2.0, 3.0, m0_ppm=-300.0)
    for f in SimEvent._fields:
        np.testing.assert_array_equal(getattr(ev, f), d["cw_" + f])
    st = Experiment.stack([Experiment(None, cw_saturation(np.linspace(-1, 1, 3), b, t, 2.8936), None, 4)
                           for b, t in ((0.5, 2.0), (1.0, 1.0))])
    for f in SimEvent._fields:
        np.testing.assert_array_equal(getattr(st.events, f), d["stack_" + f])
    pd = pad_events(ev, 5)
    for f in SimEvent._fields:
        np.testing.assert_array_equal(getattr(pd, f), d["pad_" + f])
    with pytest.raises(ValueError, match="cannot pad"):
        pad_events(ev, 1)
    assert hz_per_ppm(7.0) == pytest.approx(42.5764 * 7.0)


def test_stack_rejects_mismatched_models_and_nothing():
    a = Experiment(None, cw_saturation([0.0], 1.0, 1.0), None, 4)
    b = Experiment(None, cw_saturation([0.0], 1.0, 1.0), None, 6)
    with pytest.raises(ValueError, match="mz_loc"):
        Experiment.stack([a, b])
    with pytest.raises(ValueError, match="at least one"):
        Experiment.stack([])


@pytest.mark.parametrize("name", ["amide", "amide_noe", "amide_noe_mt", "phantom_creatine"])
def test_example_models_match_the_reference_configs(name):
    d = golden("matrix")
    i = {"amide": 0, "amide_noe": 1, "amide_noe_mt": 2, "phantom_creatine": 5}[name]
    jp = to_sim_params(example_config(name))
    for f in SimParams._fields:
        np.testing.assert_allclose(np.asarray(getattr(jp, f), float), np.asarray(d[f"m{i}_p_{f}"], float),
                                   rtol=1e-15)
    assert example_config(name).mz_loc == 2 * (1 + len(example_config(name).cest_pools))


def test_initial_state_and_padding_of_pools():
    jp = to_sim_params(example_config("amide_noe_mt"), max_cest_pools=4)
    assert np.shape(jp.cest_k) == (4,) and np.all(np.asarray(jp.cest_k)[2:] == 0)
    m = initial_state(jp, 0.6)
    op = O.Params(*[np.asarray(v) for v in jp])
    np.testing.assert_array_equal(m, O.initial_state(op, 0.6))
    with pytest.raises(ValueError, match="max_cest_pools"):
        to_sim_params(example_config("amide_noe"), max_cest_pools=1)


def test_params_layout_rows():
    jp = to_sim_params(example_config("amide_noe_mt"))
    A = pack_params(jp, 3)
    nc = 2
    assert A.shape == (13 + 5 * nc, 3)
    assert A[field_row("cest_k", 1, nc), 0] == 20.0
    assert A[field_row("cest_dw", 0, nc), 2] == 3.5
    assert A[field_row("mt_r2", None, nc), 1] == pytest.approx(1e5)
    assert A[field_row("rel_b1", None, nc), 0] == 1.0
    assert A[field_row("water_r1", None, nc), 0] == pytest.approx(1 / 1.3)
    with pytest.raises(ValueError, match="not a SimParams field"):
        field_row("nope", None, nc)


K = FreeParam("k", "cest_k", 0, scale=100.0, lo=5.0, hi=2000.0, x0=150.0)
F = FreeParam("f", "cest_f", 0, scale=0.001, lo=1e-5, hi=0.01, x0=0.0005)


def test_free_param_validation():
    with pytest.raises(ValueError, match="scope"):
        FreeParam("a", "cest_k", 0, 1, 0, 1, 0.5, scope="global")
    with pytest.raises(ValueError, match="mode"):
        FreeParam("a", "cest_k", 0, 1, 0, 1, 0.5, mode="times")
    with pytest.raises(ValueError, match="m_start"):
        FreeParam("m", "m_start", None, 1, 0, 1, 0.5, mode="add")
    with pytest.raises(ValueError, match="b0_spread"):
        FreeParam("s", "b0_spread", None, 1.0, 0.0, 1.0, 0.5, mode="factor")
    with pytest.raises(ValueError, match="frees it nowhere"):
        FreeParam("a", "cest_k", 0, 1, 0, 1, 0.5, samples=())
    assert FreeParam("a", "cest_k", 0, 1, 0, 1, 0.5, samples=(2, 0, 2)).samples == (0, 2)


def test_fit_refuses_what_it_cannot_do():
    r2w = FreeParam("r2w", "water_r2", None, 10.0, 1.0, 100.0, 14.0, scope="shared")
    exp = Experiment(to_sim_params(example_config("amide")), cw_saturation([0.0], 1.0, 1.0), None, 4)
    with pytest.raises(ValueError, match="fit_joint"):
        fit(exp, FitSpec([K, r2w]), np.zeros((2, 1)))


def test_write_params():
    jp = tile_params(to_sim_params(example_config("amide_noe")), 2)
    q = write_params(jp, np.array([[1.5, 2.0], [3.0, 4.0]]), FitSpec([K, F]))
    np.testing.assert_allclose(np.asarray(q.cest_k)[:, 0], [150.0, 300.0])
    np.testing.assert_allclose(np.asarray(q.cest_f)[:, 0], [0.002, 0.004])
    np.testing.assert_allclose(np.asarray(q.cest_k)[:, 1], [20.0, 20.0])


def test_levenberg_marquardt_without_physics():
    """tests/test_fitting.py:90-100 and tests/test_joint.py:189-197 of the reference."""
    d = golden("lm")
    resid = lambda x: np.array([10.0 * (x[1] - x[0] ** 2), 1.0 - x[0]])
    jac = lambda x: np.array([[-20.0 * x[0], 10.0], [-1.0, 0.0]])
    x, X, C = levenberg_marquardt(resid, [-1.2, 1.0], [-5.0, -5.0], [5.0, 5.0], n_iter=200, return_trajectory=True,
                                  jac_fn=jac)
    np.testing.assert_allclose(x, [1.0, 1.0], atol=1e-3)
    np.testing.assert_allclose(C[:20], d["rosen_C"][:20], rtol=1e-6, atol=1e-12)
    r = lambda x: np.array([x[0] - 1.0, x[1] - 2.0, 0.1 * x[0] * x[1]])
    held = levenberg_marquardt(r, [0.0, 5.0], [-10, -10], [10, 10], n_iter=30, free=[1.0, 0.0])
    assert held[1] == 5.0
    both = levenberg_marquardt(r, [0.0, 5.0], [-10, -10], [10, 10], n_iter=30)
    ones = levenberg_marquardt(r, [0.0, 5.0], [-10, -10], [10, 10], n_iter=30, free=[1.0, 1.0])
    np.testing.assert_array_equal(both, ones)


def test_spread_nodes_and_weights():
    """tests/test_joint.py:285-294 of the reference."""
    u, w = B0Spread(shape="gauss", nodes=5).nodes_weights()
    assert w.sum() == pytest.approx(1.0) and np.sum(w * u ** 2) == pytest.approx(1.0)
    u, w = B0Spread(shape="lorentz", nodes=9, cut=20.0).nodes_weights()
    T = np.arctan(20.0)
    assert np.sum(w / (1 + u ** 2)) == pytest.approx(0.5 + np.sin(2 * T) / (4 * T), rel=1e-10)
    with pytest.raises(ValueError, match="shape"):
        B0Spread(shape="box")
