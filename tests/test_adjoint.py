"""The adjoint kernel: every tangent of a single-event table (CW Z-spectra and B1 ladders,
sequences/saturation.py:28-84) from one Frechet derivative of the event's exponential, against forward
mode (one dual-number launch per tangent, the chain kernel) and the oracle's exact forward derivatives.
The work counters show which kernel ran: forward mode counts the dense squarings once per launch, the
adjoint kernel once."""
import numpy as np
import pytest

import bmc_oracle as O

pytestmark = pytest.mark.gpu


def _batch(n, nc, seed, mt=True):
    rng = np.random.default_rng(seed)
    dws = np.array([3.5, 2.0, 1.0, -3.5, 1.9, -1.6])[:nc]
    return O.Params(
        water_r1=1.0 / rng.uniform(0.8, 2.5, n), water_r2=1.0 / rng.uniform(0.03, 0.12, n), water_f=np.ones(n),
        cest_k=rng.uniform(10, 5000, (n, nc)), cest_f=rng.uniform(1e-5, 0.02, (n, nc)),
        cest_dw=np.broadcast_to(dws, (n, nc)).copy(), cest_r1=np.ones((n, nc)),
        cest_r2=np.broadcast_to(np.array([10.0, 30.0, 50.0, 200.0, 30.0, 40.0])[:nc], (n, nc)).copy(),
        mt_k=np.full(n, 30.0 if mt else 0.0), mt_f=np.full(n, 0.05 if mt else 0.0), mt_dw=np.full(n, -2.5),
        mt_r1=np.ones(n), mt_r2=np.full(n, 1e5), mt_lineshape=np.full(n, 2 if mt else 0), b0=np.full(n, 3.0),
        gamma=np.full(n, 267.5153), b0_inhom=rng.uniform(-0.3, 0.3, n), rel_b1=rng.uniform(0.8, 1.2, n))


def _ladder(n_ppm=9, b1s=(0.7, 3.0), m0_ppm=-300.0):
    return O.stack_events([O.cw_saturation(np.linspace(-6, 6, n_ppm), b1, 2.0, 3.0, m0_ppm=m0_ppm) for b1 in b1s])


def _slots(nc, mt):
    s = [("water_r2", None), ("b0_inhom", None), ("rel_b1", None), ("water_r1", None)]
    if nc:
        s = [("cest_k", 0), ("cest_f", nc - 1)] + s
    if mt:
        s.append(("mt_r2", None))            # the super-Lorentzian's own derivative
    return s


def _jvp(pb, ev, m0, nc, slots, seeds, dm0=None, spread=None, mode="auto"):
    """(z, jz, work counters) from bmc_simulate_jvp_counted in the given tangent mode."""
    import torch
    from bmc_b200 import _lib, settings
    from bmc_b200.fitting import field_row
    from bmc_b200.simulation import DeviceEvents, SimEvent, SimParams, _device, pack_params, problem
    n = m0.shape[0]
    n_off, n_ev = np.asarray(ev.type).shape
    settings.use_tangents(mode)
    try:
        dev_ev = DeviceEvents(SimEvent(*ev))
        pdev = _device(pack_params(SimParams(*pb), n))
        mdev = _device(m0)
        P = len(slots)
        tg = _lib.Tangents()
        tg.n_tangents = P
        for i, (f, ix) in enumerate(slots):
            tg.field_row[i] = _lib.SEED_SPREAD_SIGMA if f == "sigma" else field_row(f, ix, nc)
        sd = _device(seeds)
        tg.d_seed = sd.data_ptr()
        dd = _device(dm0) if dm0 is not None else None
        tg.d_dm0 = dd.data_ptr() if dd is not None else None
        z = torch.empty((n, n_off), dtype=torch.float64, device="cuda")
        jz = torch.empty((P, n, n_off), dtype=torch.float64, device="cuda")
        work = torch.zeros(5, dtype=torch.int64, device="cuda")
        sp, keep = (None, None) if spread is None else spread
        pr = problem(n, n_off, n_ev, nc, O.mz_loc(nc), _lib.F64)
        _lib.check(_lib.lib().bmc_simulate_jvp_counted(pr, _lib.ptr(pdev), dev_ev.struct, _lib.ptr(mdev), sp, tg,
                                                       _lib.ptr(z), _lib.ptr(jz), _lib.ptr(work),
                                                       _lib.stream_handle()))
        torch.cuda.synchronize()
        return z.cpu().numpy(), jz.cpu().numpy(), work.cpu().numpy()
    finally:
        settings.use_tangents("auto")


def _launches(nc, P):
    return (P + 1) // 2 if nc <= 1 else P


@pytest.mark.parametrize("nc,mt", [(0, True), (1, True), (2, False), (3, True), (4, True), (4, False), (5, True)])
def test_adjoint_tangents_equal_forward_mode(cuda, nc, mt):
    """Six or seven tangents of every kind (exchange, fraction, relaxation, B0, B1, the MT lineshape),
    per-voxel seeds and start-state tangents, two B1 rungs and the unsaturated reference offset."""
    n = 6
    pb = _batch(n, nc, seed=100 + nc, mt=mt)
    ev = _ladder()
    N = 3 * nc + 4
    m0 = np.stack([O.initial_state(O.sample(pb, i)) for i in range(n)])
    slots = _slots(nc, mt)
    P = len(slots)
    rng = np.random.default_rng(nc)
    seeds = rng.normal(size=(P, n))
    dm0 = np.zeros((P, n, N))
    dm0[0] = rng.normal(size=(n, N)) * 0.1
    za, ja, wa = _jvp(pb, ev, m0, nc, slots, seeds, dm0, mode="auto")
    zf, jf, wf = _jvp(pb, ev, m0, nc, slots, seeds, dm0, mode="forward")
    np.testing.assert_allclose(za, zf, rtol=0, atol=1e-13)
    for p in range(P):
        np.testing.assert_allclose(ja[p], jf[p], rtol=1e-9, atol=1e-11 * max(1.0, np.abs(jf[p]).max()),
                                   err_msg=f"tangent {slots[p]}")
    assert wa[2] > 0 and wf[2] == _launches(nc, P) * wa[2]      # one launch against one per tangent (pair)


def test_adjoint_with_a_b0_spread_and_its_width(cuda):
    """Three isochromats per voxel, the spread width among the tangents."""
    from bmc_b200 import _lib
    from bmc_b200.simulation import B0Spread, _device
    nc, n = 1, 5
    pb = _batch(n, nc, seed=7)
    ev = _ladder(n_ppm=7)
    m0 = np.stack([O.initial_state(O.sample(pb, i)) for i in range(n)])
    slots = [("sigma", None), ("cest_k", 0), ("b0_inhom", None)]
    seeds = np.random.default_rng(1).normal(size=(3, n))
    u, w = B0Spread(nodes=3).nodes_weights()
    sig = _device(np.linspace(5.0, 20.0, n))
    spread = _lib.spread_struct(u, w, sig)
    za, ja, wa = _jvp(pb, ev, m0, nc, slots, seeds, spread=spread, mode="auto")
    zf, jf, wf = _jvp(pb, ev, m0, nc, slots, seeds, spread=spread, mode="forward")
    np.testing.assert_allclose(za, zf, rtol=0, atol=1e-13)
    np.testing.assert_allclose(ja, jf, rtol=1e-9, atol=1e-11 * np.abs(jf).max())
    assert wf[2] == 2 * wa[2]


def test_adjoint_jacobian_matches_the_oracle(cuda):
    """Water + 4 CEST pools + super-Lorentzian MT on the fit ladder: five tangents against the oracle's
    exact forward mode (Pade-13 exponentials, float64)."""
    from bmc_b200.design import jacobian
    from bmc_b200.fitting import Experiment, FitSpec, FreeParam
    from bmc_b200.simulation import SimEvent, SimParams
    nc = 4
    p1 = O.sample(_batch(1, nc, seed=11), 0)
    ev = _ladder(n_ppm=11, b1s=(0.5, 2.0))
    m0 = O.initial_state(p1)
    slots = [("cest_k", 0), ("cest_f", 1), ("water_r2", None), ("b0_inhom", None), ("mt_r2", None)]
    xs = [float(np.atleast_1d(getattr(p1, f))[0 if i is None else i]) for f, i in slots]
    spec = FitSpec([FreeParam(f"a{j}", f, i, 1.0, -1e9, 1e9, x) for j, ((f, i), x) in enumerate(zip(slots, xs))])
    Z, J = jacobian(Experiment(SimParams(*p1), SimEvent(*ev), m0, O.mz_loc(nc)), spec, xs)
    Zo, Jo = O.spectrum_jacobian(p1, ev, m0, [O.Slot(f, i) for f, i in slots])
    np.testing.assert_allclose(Z, Zo, rtol=0, atol=1e-10)
    np.testing.assert_allclose(J, Jo, rtol=1e-7, atol=1e-9 * max(1.0, np.abs(Jo).max()))


def test_lm_fit_takes_the_same_steps_in_both_modes(cuda):
    """README.md:62-94's ladder fit (bmc_lm_fit): the adjoint Jacobians give forward mode's iterates."""
    from bmc_b200 import settings
    from bmc_b200.configs import example_config
    from bmc_b200.fitting import Experiment, FitSpec, FreeParam, fit
    from bmc_b200.sequences import cw_saturation
    from bmc_b200.simulation import initial_state, to_sim_params
    params = example_config("amide")
    jp = to_sim_params(params)
    m0 = initial_state(jp)
    ppm = np.linspace(-6, 6, 61)
    ladder = Experiment.stack([Experiment(jp, cw_saturation(ppm, b, 2.0, params.system.b0), m0, params.mz_loc)
                               for b in (0.5, 1.0, 2.0, 4.0)])
    z = ladder.simulate()
    z = z[None, :] + 0.002 * np.random.default_rng(3).standard_normal((1, z.size))
    spec = FitSpec([FreeParam("k", "cest_k", 0, scale=100.0, lo=5.0, hi=5000.0, x0=300.0),
                    FreeParam("f", "cest_f", 0, scale=0.001, lo=1e-6, hi=0.05, x0=0.0005)])
    out = {}
    for mode in ("auto", "forward"):
        settings.use_tangents(mode)
        try:
            out[mode] = fit(ladder, spec, z, n_per_block=len(ppm), n_iter=15)
        finally:
            settings.use_tangents("auto")
    np.testing.assert_allclose(out["auto"].x, out["forward"].x, rtol=1e-9)
    np.testing.assert_allclose(out["auto"].rms, out["forward"].rms, rtol=1e-9)


def test_pulse_trains_stay_in_forward_mode(cuda):
    """Rows whose state evolves in many events (pulse samples, gaps, recovery) keep the chain kernel:
    the automatic mode's results are forward mode's, bit for bit."""
    nc, n = 2, 3
    pb = _batch(n, nc, seed=5)
    t = np.array([1] * 6 + [0, 4, 0, 3], np.int32)
    dt = np.array([0.005] * 6 + [0.002, 0.0, 1.0, 0.0])
    amp = np.array([40.0] * 6 + [0.0] * 4)
    n_off = 4
    freq = np.linspace(-3, 3, n_off)[:, None] * 127.7 * (t[None, :] == 1)
    ev = O.Events(np.tile(t, (n_off, 1)), np.tile(dt, (n_off, 1)), np.tile(amp, (n_off, 1)),
                  np.zeros((n_off, t.size)), freq, np.tile(np.int32([-1] * 9 + [0]), (n_off, 1)))
    m0 = np.stack([O.initial_state(O.sample(pb, i)) for i in range(n)])
    slots = [("cest_k", 0), ("water_r2", None), ("b0_inhom", None)]
    seeds = np.ones((3, n))
    za, ja, wa = _jvp(pb, ev, m0, nc, slots, seeds, mode="auto")
    zf, jf, wf = _jvp(pb, ev, m0, nc, slots, seeds, mode="forward")
    np.testing.assert_array_equal(za, zf)
    np.testing.assert_array_equal(ja, jf)
    np.testing.assert_array_equal(wa, wf)


# ------------------------------------------------------------------------------------------------
# uneven batches: the block kernel (rows = a block of pulse and gap repeated r times, then the readout)
# ------------------------------------------------------------------------------------------------
def _block_table(ppm, b1s, n_pulses, tp=0.05, gap=0.005, b0=3.0):
    from bmc_b200.simulation import SimEvent
    rows = [(b, p) for b in b1s for p in ppm]
    n, ne = len(rows), 2 * n_pulses + 1
    return SimEvent(np.tile(np.int32([1, 0] * n_pulses + [3]), (n, 1)),
                    np.tile([tp, gap] * n_pulses + [0.0], (n, 1)),
                    np.array([[b * 267.5153 / (2 * np.pi), 0.0] * n_pulses + [0.0] for b, _ in rows]),
                    np.zeros((n, ne)),
                    np.array([[p * 42.5764 * b0, 0.0] * n_pulses + [0.0] for _, p in rows]),
                    np.tile(np.int32([-1] * (ne - 1) + [0]), (n, 1)))


def _uneven_tangents(g, slots, nc, seeds, dm0, mode):
    import torch
    from bmc_b200 import _lib, settings
    from bmc_b200.fitting import field_row
    P = len(slots)
    tg = _lib.Tangents()
    tg.n_tangents = P
    for i, (f, ix) in enumerate(slots):
        tg.field_row[i] = field_row(f, ix, nc)
    tg.d_seed, tg.d_dm0 = seeds.data_ptr(), dm0.data_ptr()
    settings.use_tangents(mode)
    try:
        jz = torch.empty((P, g.n_chains), dtype=torch.float64, device="cuda")
        z = g.plan.run(g.params, g.m0, tg, jz)
        torch.cuda.synchronize()
        return z.cpu().numpy(), jz.cpu().numpy()
    finally:
        settings.use_tangents("auto")


@pytest.mark.parametrize("nc,mt", [(1, False), (2, True), (4, False), (5, True)])
def test_uneven_block_tangents_equal_forward_mode(cuda, nc, mt):
    """Voxels of one pool count with trains of 1, 2, 7 and 40 block pulses (no block, and blocks of 2 to
    40 repeats), seven tangents of every kind with per-voxel seeds and a start-state tangent: the block
    kernel against forward mode (one chain-kernel launch per tangent)."""
    import torch
    from bmc_b200.fitting import Experiment
    from bmc_b200.simulation import SimParams
    from bmc_b200.uneven import UnevenBatch
    rng = np.random.default_rng(50 + nc)
    tables = [_block_table(np.linspace(-5, 5, 7), (0.8, 2.5), n) for n in (1, 2, 7, 40)]
    pb = _batch(8, nc, seed=60 + nc, mt=mt)
    exps = [Experiment(SimParams(*O.sample(pb, i)), tables[i % 4], O.initial_state(O.sample(pb, i)), O.mz_loc(nc))
            for i in range(8)]
    g = UnevenBatch(exps).groups[0]
    slots = [("cest_k", 0), ("cest_f", nc - 1), ("water_r2", None), ("water_r1", None), ("b0_inhom", None),
             ("rel_b1", None), ("mt_k" if mt else "cest_r2", None if mt else 0)]
    P, nv, N = len(slots), len(g.voxels), 3 * nc + 4
    seeds = torch.as_tensor(rng.normal(size=(P, nv))).cuda()
    dm0 = torch.zeros((P, nv, N), dtype=torch.float64, device="cuda")
    dm0[2] = torch.as_tensor(rng.normal(size=(nv, N)) * 0.1)
    za, ja = _uneven_tangents(g, slots, nc, seeds, dm0, "auto")
    zf, jf = _uneven_tangents(g, slots, nc, seeds, dm0, "forward")
    np.testing.assert_allclose(za, zf, rtol=0, atol=1e-12)
    for p in range(P):
        np.testing.assert_allclose(ja[p], jf[p], rtol=1e-8, atol=1e-10 * max(1.0, np.abs(jf[p]).max()),
                                   err_msg=f"tangent {slots[p]}")
