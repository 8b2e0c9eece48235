"""The learned warm start, end to end on the GPU: a network trained on simulated ladders predicts
starting values close to the truth, and the LM fit started there reaches the truth in fewer
iterations than the plain fit from the fixed x0 -- the gain the network brings. The plain fit stays
the fallback, so the warm-started result is never worse than the plain one on the same data.

Model: configuration 1's water + amide pool at 3 T, its ladder (4 x 61 CW offsets, 2 s), free (k, f)
drawn uniformly from k in [20, 1000] 1/s, f in [3e-4, 3e-3]; noise-free held-out voxels.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained(cuda):
    from bmc_b200.configs import example_config
    from bmc_b200.fitting import Experiment, FitSpec, FreeParam
    from bmc_b200.sequences import cw_saturation
    from bmc_b200.simulation import initial_state, to_sim_params
    from bmc_b200.warmstart import LadderWarmStart
    p = example_config("amide")
    jp = to_sim_params(p)
    ppm = np.linspace(-6.0, 6.0, 61)
    ladder = Experiment.stack([Experiment(jp, cw_saturation(ppm, b, 2.0, 3.0), initial_state(jp), p.mz_loc)
                               for b in (0.5, 1.0, 2.0, 4.0)])
    spec = FitSpec([FreeParam("k", "cest_k", 0, 100.0, 5.0, 5000.0, 300.0),
                    FreeParam("f", "cest_f", 0, 1e-3, 1e-6, 0.05, 5e-4)])
    ws = LadderWarmStart(ladder, spec, ranges=[(20.0, 1000.0), (3e-4, 3e-3)], sigma=0.002, seed=1)
    hist = ws.train(n_train=65536, epochs=20, batch=1024, lr=1e-3, seed=1)
    X = ws.draw(1024, seed=77)
    z = ws.simulate64(X)
    return ws, ladder, spec, hist, X, z


def _ok(x, X):
    return np.all(np.abs(x / X - 1.0) <= 0.01, axis=1)


def test_training_converges(trained):
    ws, _, _, hist, _, _ = trained
    assert hist[-1] < 0.2 * hist[0], hist
    assert ws.mlp.status(1024) == 0


def test_network_starting_values_beat_the_fixed_start(trained):
    ws, _, spec, _, X, z = trained
    x0 = ws.starting_values(z)
    err_net = np.median(np.abs(x0 / X - 1.0), axis=0)
    err_fixed = np.median(np.abs(spec.x0_phys / X - 1.0), axis=0)
    assert (err_net < 0.3 * err_fixed).all(), (err_net, err_fixed)
    assert (x0 >= spec.lo_phys).all() and (x0 <= spec.hi_phys).all()


def test_warm_start_needs_fewer_iterations(trained):
    from bmc_b200.fitting import fit
    ws, ladder, spec, _, X, z = trained
    plain3 = fit(ladder, spec, z, n_iter=3)
    warm3 = fit(ladder, spec, z, n_iter=3, x0_phys=ws.starting_values(z))
    plain30 = fit(ladder, spec, z, n_iter=30)
    f_plain3, f_warm3, f_plain30 = _ok(plain3.x, X).mean(), _ok(warm3.x, X).mean(), _ok(plain30.x, X).mean()
    assert f_warm3 > f_plain3 + 0.2, (f_warm3, f_plain3)
    # with the plain fallback, a short warm fit is as good as the full plain fit
    res = ws.fit(z, n_iter_warm=4, n_iter_plain=30, fallback_rms=1e-6)     # noise-free: converged rms ~1e-10
    assert _ok(res.x, X).mean() >= f_plain30 - 0.01, (_ok(res.x, X).mean(), f_plain30)
    assert (res.rms <= np.maximum(plain30.rms, 1e-6) * (1 + 1e-6) + 1e-12).mean() > 0.99
