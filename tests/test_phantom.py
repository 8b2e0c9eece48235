"""The reference's phantom tutorials on the shipped measurement, through the public API, against the
float64 oracle LM on the same data.

Tutorial 08 (examples/08_quesp.py:66-85): k, f and pool T2 of a tube from its QUESP ladder (8 B1 rungs of
the scanner's 4,041-event pulse trains). Tutorial 10 (examples/10_shared_water.py:94-101): the joint fit
with a water-R2 factor, M_start and a B0-spread width shared by the tubes. To keep the oracle's share
short, the tests fit a subset of the data -- every fourth offset with |ppm| >= 1, one tube for tutorial
08, three tubes, two rungs and a 3-node spread for tutorial 10 -- and both sides fit exactly that subset
from the same start. The oracle: residuals from the float64 C restatement (Pade-13 expm per event), the
Jacobian by central differences of those residuals, and the reference's LM schedule (fitting/lm.py:43-61,
fitting/joint.py:149-162 for the joint step). Fitted values agree to 1e-3 relative."""
import numpy as np
import pytest

import bmc_oracle as O

pytestmark = pytest.mark.gpu


def _keep(d):
    keep = np.abs(d["ppm"]) >= 1.0
    return keep & (np.arange(keep.size) % 4 == 0)


def _stems(rungs):
    return [f"quesp_sim_b1_{('%g' % b).replace('.', 'p')}uT" for b in rungs]


def _ladder(d, tubes, rungs):
    """(Experiment of the tubes, measured Z, offsets per rung) as tutorials 08-10 build them."""
    import bench
    from bmc_b200.fitting import Experiment
    from bmc_b200.simulation import SimParams, initial_state
    p = bench.phantom_params(d)
    p = SimParams(*[np.asarray(v)[tubes] for v in p])
    m0 = np.stack([initial_state(SimParams(*[np.asarray(v)[i] for v in p]), float(d["m_start"]))
                   for i in range(len(tubes))])
    keep = _keep(d)
    lad = Experiment.stack([Experiment(p, bench.phantom_events(s, keep), m0, 4) for s in _stems(rungs)])
    ri = [list(d["b1_levels_uT"]).index(b) for b in rungs]
    z = d["Z_quesp"][tubes][:, ri][:, :, keep].reshape(len(tubes), -1).astype(np.float64)
    return lad, z, int(keep.sum())


def _oracle_z(p_soa, ev, m0):
    return O.c_simulate_z(p_soa, O.Events(*[np.asarray(a) for a in ev]), m0, 1, 4)


def _central_jacobian(resid, x, rel=1e-6):
    r0 = resid(x)
    J = np.empty((r0.size, x.size))
    for j in range(x.size):
        h = rel * max(1.0, abs(x[j]))
        e = np.zeros_like(x)
        e[j] = h
        J[:, j] = (resid(x + e) - resid(x - e)) / (2 * h)
    return r0, J


def _slots():
    from bmc_b200.fitting import FreeParam
    K = FreeParam("k", "cest_k", 0, scale=1000.0, lo=5.0, hi=2000.0, x0=300.0)
    F = FreeParam("f", "cest_f", 0, scale=0.01, lo=1e-5, hi=0.03, x0=0.008)
    T2 = FreeParam("r2p", "cest_r2", 0, scale=100.0, lo=10.0, hi=1000.0, x0=100.0)
    return K, F, T2


def test_tutorial08_fit_matches_the_oracle_lm(cuda):
    import bench
    from bmc_b200.fitting import FitSpec, fit
    from bmc_b200.simulation import pack_params
    d = bench.phantom_data("pool")
    tube, n_iter = 2, 12                                     # creatine pH 7.51: a fast-exchanging amine
    rungs = list(d["b1_levels_uT"])
    lad, z, n_per = _ladder(d, [tube], rungs)
    spec = FitSpec(list(_slots()))
    res = fit(lad, spec, z, n_iter=n_iter, n_per_block=n_per)

    base = pack_params(lad.params, 1)
    rows = [3, 4, 3 + 4]                                     # cest_k, cest_f, cest_r2 rows for one pool
    sc = spec.scales

    def resid(xs):
        p = base.copy()
        p[rows, 0] = xs * sc
        return _oracle_z(p, lad.events, lad.m0)[0] - z[0]

    rj = lambda xs, need_jac=True: _central_jacobian(resid, xs) if need_jac else (resid(xs), None)
    x = O.levenberg_marquardt(rj, spec.x0_phys / sc, spec.lo_phys / sc, spec.hi_phys / sc, n_iter=n_iter)
    print("gpu", res.x[0], "oracle", x * sc, "rms/noise", res.rms[0] / d["noise_quesp"][tube])
    np.testing.assert_allclose(res.x[0], x * sc, rtol=1e-3)
    assert res.rms[0] < 5 * d["noise_quesp"][tube]


def test_tutorial10_joint_fit_matches_the_dense_oracle_lm(cuda):
    import bench
    from dataclasses import replace
    from bmc_b200.fitting import FitSpec, FreeParam, fit_joint
    from bmc_b200.simulation import B0Spread, pack_params
    d = bench.phantom_data()
    tubes = [0, 3, 5]                                        # PBS (no pool), creatine, carnosine
    rungs = [0.5, 1.5]
    n_iter = 4
    lad, z, n_per = _ladder(d, tubes, rungs)
    pool = (1, 2)
    K, F, T2 = (replace(s, samples=pool) for s in _slots())
    R2F = FreeParam("r2w", "water_r2", None, scale=1.0, lo=0.5, hi=2.0, x0=1.0, scope="shared", mode="factor")
    MS = FreeParam("m_start", "m_start", None, scale=1.0, lo=0.2, hi=1.0, x0=0.6, scope="shared")
    SIG = FreeParam("sigma", "b0_spread", None, scale=10.0, lo=0.0, hi=8.0, x0=5.0, scope="shared")
    spec = FitSpec([K, F, T2, R2F, MS, SIG])
    x0 = np.tile([s.x0 for s in spec.slots], (3, 1))
    x0[1:, :3] = [[400.0, 0.004, 80.0], [250.0, 0.0008, 60.0]]
    spread = B0Spread(nodes=3)
    res = fit_joint(lad, spec, z, n_iter=n_iter, n_per_block=n_per, x0_phys=x0, spread=spread)

    # the dense oracle: columns k1, k2, f1, f2, r2p1, r2p2, r2w factor, m_start, sigma (scaled units)
    base = pack_params(lad.params, 3)
    u, w = spread.nodes_weights()
    row = {"k": 3, "f": 4, "r2p": 7, "r2w": 1, "wf": 2, "b0i": 16, "gamma": 15, "b0": 14}   # one CEST pool
    scl = np.array([1000.0, 1000.0, 0.01, 0.01, 100.0, 100.0, 1.0, 1.0, 10.0])

    def model(xs):
        xp = xs * scl
        p = base.copy()
        for j, i in enumerate(pool):
            p[row["k"], i], p[row["f"], i], p[row["r2p"], i] = xp[j], xp[2 + j], xp[4 + j]
        p[row["r2w"]] = base[row["r2w"]] * xp[6]
        m0 = np.zeros((3, 7))                                # water z, pool z: their fractions (no MT)
        m0[:, 4] = p[row["wf"]]
        m0[:, 5] = p[row["f"]]
        m0 *= xp[7]                                          # m_start rebuilt from the current pools
        g = p[row["gamma"]] * p[row["b0"]] / (2 * np.pi)    # Hz per ppm
        zs = 0.0
        for uj, wj in zip(u, w):
            q = p.copy()
            q[row["b0i"]] = p[row["b0i"]] + uj * xp[8] / g
            zs = zs + wj * _oracle_z(q, lad.events, m0)
        return zs

    def resid(xs):
        return (model(xs) - z).reshape(-1)

    lo = np.array([5, 5, 1e-5, 1e-5, 10, 10, 0.5, 0.2, 0.0]) / scl
    hi = np.array([2000, 2000, 0.03, 0.03, 1000, 1000, 2.0, 1.0, 8.0]) / scl
    x = np.array([400.0, 250.0, 0.004, 0.0008, 80.0, 60.0, 1.0, 0.6, 5.0]) / scl
    lam = 1e-2
    for _ in range(n_iter):
        r, J = _central_jacobian(resid, x)
        c = float(r @ r)
        xn = O.lm_trial(x, lam, J, r, lo, hi)
        cn = float(resid(xn) @ resid(xn))
        if cn < c:
            x, lam = xn, lam * 0.5
        else:
            lam *= 3.0
    xp = x * scl
    got = np.concatenate([res["k"][1:], res["f"][1:], res["r2p"][1:],
                          [res["r2w"][0], res["m_start"][0], res["sigma"][0]]])
    print("gpu", got, "oracle", xp)
    np.testing.assert_allclose(got, xp, rtol=1e-3)
    assert not res.free[0, :3].any() and res["k"][0] == 0.0   # the PBS tube keeps its carried pool values
