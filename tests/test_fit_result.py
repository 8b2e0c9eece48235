"""FitResult, the joint-fit column map and the error bars, on the host (no GPU).

The error bars of a coupled joint fit are assembled from every sample's local normal matrix; here they
are checked against the dense form of fitting/joint.py:418-453 (pinv of J^T J of the full joint
Jacobian, misfit-scaled) on random Jacobians, and the independent-sample form likewise per sample."""
import numpy as np
import pytest

from bmc_b200.fitting import FitResult, FitSpec, FreeParam, _columns, _error_bars
from bmc_b200.design import CRLB


def _spec():
    return FitSpec([FreeParam("k", "cest_k", 0, 100.0, 5.0, 5000.0, 300.0),
                    FreeParam("f", "cest_f", 0, 1e-3, 1e-6, 0.05, 5e-4, samples=(0, 2)),
                    FreeParam("r2", "water_r2", None, 10.0, 1.0, 100.0, 14.0, scope="shared"),
                    FreeParam("b1", "rel_b1", None, 1.0, 0.7, 1.3, 1.0, scope="block", mode="factor")])


def test_column_map():
    lay = _columns(_spec(), 3, 2)
    assert lay.n_loc == 5 and list(lay.pos) == [0, 1, 2, 3]
    # k per sample (3), f in samples 0 and 2 (2), r2 shared (1), b1 per experiment (2)
    assert [c[0] for c in lay.cols] == [0, 0, 0, 1, 1, 2, 3, 3]
    assert lay.col_of[1].tolist() == [1, -1, 5, 6, 7]
    assert lay.free.tolist() == [[True, True, True, True], [True, False, True, True], [True, True, True, True]]
    with pytest.raises(ValueError, match="do not exist"):
        _columns(FitSpec([FreeParam("f", "cest_f", 0, 1e-3, 0, 1, 0, samples=(0, 5))]), 3, 1)


def _dense_bars(J, r, scale):
    """The dense reference form: cov = pinv(J^T J) s^2, sd = sqrt(diag) * scale, corr."""
    s2 = float(r @ r) / max(r.size - J.shape[1], 1)
    cov = np.linalg.pinv(J.T @ J) * s2
    sd = np.sqrt(np.clip(np.diag(cov), 0, None))
    return sd * scale, cov / np.outer(sd, sd)


def test_coupled_error_bars_equal_the_dense_form():
    spec = _spec()
    n, nb, n_pts = 3, 2, 14
    lay = _columns(spec, n, nb)
    rng = np.random.default_rng(4)
    Jl = rng.normal(size=(n, n_pts, lay.n_loc))
    r = rng.normal(scale=1e-3, size=(n, n_pts))
    x = rng.uniform(0.5, 2.0, len(lay.cols))
    sd, corr, blocks = _error_bars(np.einsum("inj,ink->ijk", Jl, Jl), r, lay, spec, True, x)
    P = len(lay.cols)
    J = np.zeros((n, n_pts, P))
    for p, (l, who, b) in enumerate(lay.cols):
        for i in who:
            J[i, :, p] = Jl[i, :, lay.pos[l] + max(b, 0)]
    scale = spec.scales[[l for l, _, _ in lay.cols]]
    sd_d, corr_d = _dense_bars(J.reshape(-1, P), r.reshape(-1), scale)
    for p, (l, who, b) in enumerate(lay.cols):
        if b >= 0:
            continue
        for i in who:
            assert sd[i, l] == pytest.approx(sd_d[p], rel=1e-9)
    i = 2                                              # k, f, r2 of sample 2: columns 2, 4, 5
    np.testing.assert_allclose(corr[i][np.ix_([0, 1, 2], [0, 1, 2])], corr_d[np.ix_([2, 4, 5], [2, 4, 5])],
                               rtol=1e-9)
    assert np.isnan(sd[1, 1]) and np.isnan(sd[:, 3]).all()       # held f of sample 1; b1 lives in blocks
    np.testing.assert_allclose(blocks["b1"]["sd"], sd_d[6:8], rtol=1e-9)
    np.testing.assert_allclose(blocks["b1"]["x"], x[6:8] * 1.0)


def test_independent_error_bars_equal_the_dense_form():
    spec = FitSpec([FreeParam("k", "cest_k", 0, 100.0, 5.0, 5000.0, 300.0),
                    FreeParam("f", "cest_f", 0, 1e-3, 1e-6, 0.05, 5e-4, samples=(1,))])
    lay = _columns(spec, 2, 1)
    rng = np.random.default_rng(5)
    Jl = rng.normal(size=(2, 9, 2))
    r = rng.normal(scale=1e-3, size=(2, 9))
    sd, corr, blocks = _error_bars(np.einsum("inj,ink->ijk", Jl, Jl), r, lay, spec, False)
    sd0, _ = _dense_bars(Jl[0][:, :1], r[0], spec.scales[:1])
    sd1, corr1 = _dense_bars(Jl[1], r[1], spec.scales)
    assert sd[0, 0] == pytest.approx(sd0[0], rel=1e-10) and np.isnan(sd[0, 1])
    np.testing.assert_allclose(sd[1], sd1, rtol=1e-10)
    np.testing.assert_allclose(corr[1], corr1, rtol=1e-10)
    assert blocks == {}


def test_fit_result_views():
    spec = FitSpec([FreeParam("k", "cest_k", 0, 100.0, 5.0, 5000.0, 300.0),
                    FreeParam("f", "cest_f", 0, 1e-3, 1e-6, 0.05, 5e-4)])
    x = np.array([[5.0, 1e-3], [250.0, 0.05], [300.0, 4e-4]])
    z_meas = np.zeros((3, 6))
    z_fit = np.tile([0.0, 0.0, 0.0, 3.0, 3.0, 3.0], (3, 1))
    free = np.array([[True, True], [True, False], [True, True]])
    res = FitResult(x, z_fit, z_meas, spec, n_per_block=3, free=free, x0=np.array([[5.0, 2e-3], [1.0, 0.05],
                                                                                   [300.0, 4e-4]]))
    assert res.at_bounds.tolist() == [[True, False], [False, False], [False, False]]   # held f of 1 not railed
    assert res.unmoved.tolist() == [[True, False], [False, False], [True, True]]
    np.testing.assert_allclose(res.rms, np.sqrt(4.5))
    np.testing.assert_allclose(res.rms_per_block, [[0.0, 3.0]] * 3)
    np.testing.assert_array_equal(res["k"], x[:, 0])
    with pytest.raises(KeyError, match="no parameter"):
        res["t2"]
    text = res.summary()
    assert "[b]" in text and "[h]" in text and "on a bound" in text
    assert "1 values on a bound" in repr(res)
    plain = FitResult(x[2:], z_fit[2:], z_meas[2:], spec)
    assert plain.unmoved is None and plain.rms_per_block is None and "[b]" not in plain.summary()


def test_crlb_views():
    b = CRLB(("k", "f"), np.array([100.0, -2e-3]), np.array([5.0, 1e-4]), np.eye(2), np.eye(2), np.zeros((3, 2)))
    np.testing.assert_allclose(b.rel_sd, [0.05, 0.05])
    assert b["f"] == 1e-4
    with pytest.raises(ValueError):
        b["t2"]
    assert "5.00% of the value" in b.summary()
