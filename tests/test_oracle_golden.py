"""The oracle against golden vectors produced by the reference's own source (tests/golden).

tests/golden/make_golden.py executes BMC-JAX's Python (matrix build, time step, scan, spread,
event builders, LM, fit) in float64 and stores inputs and outputs; these tests pin the CPU oracle
to them. CPU only.
"""
import numpy as np
import pytest

import bmc_oracle as O
from conftest import golden, unpack_params, unpack_events


def test_system_matrices_match_the_reference_bit_for_bit():
    d = golden("matrix")
    i = 0
    while f"m{i}_A" in d:
        p = unpack_params(d, f"m{i}_p_", O.Params)
        a, ph, fr = d[f"m{i}_rf"]
        A, C = O.bmc_system(p, a, ph, fr)
        np.testing.assert_array_equal(A, d[f"m{i}_A"])
        np.testing.assert_array_equal(C, d[f"m{i}_C"])
        i += 1
    assert i >= 6


SPECTRA = ["readme", "mt_sl", "mt_lor", "creatine", "semantics", "front_pad", "tail_pad"]


@pytest.mark.parametrize("tag", SPECTRA)
def test_spectra_match_the_reference(tag):
    d = golden("spectra")
    p = unpack_params(d, f"{tag}_p_", O.Params)
    ev = unpack_events(d, f"{tag}_e_", O.Events)
    M = O.simulate_spectrum(p, ev, d[f"{tag}_m0"])
    np.testing.assert_allclose(M, d[f"{tag}_M"], rtol=0, atol=1e-12)


def test_pulsed_train_matches_the_reference():
    """The shipped 4041-event QUESP train (RF samples with phases, spoilers, gaps, recovery, ADC)."""
    d = golden("spectra")
    p = unpack_params(d, "quesp_p_", O.Params)
    ev = unpack_events(d, "quesp_e_", O.Events)
    ev = O.Events(*[np.asarray(a)[:2] for a in ev])          # two offsets keep this test short
    M = O.simulate_spectrum(p, ev, d["quesp_m0"])
    np.testing.assert_allclose(M, d["quesp_M"][:2], rtol=0, atol=1e-12)


@pytest.mark.parametrize("tag,shape,nodes", [("gauss5", "gauss", 5), ("lorentz3", "lorentz", 3)])
def test_spread_matches_the_reference(tag, shape, nodes):
    d = golden("spread")
    u, w = O.spread_nodes(shape, nodes)
    np.testing.assert_allclose(u, d[f"{tag}_u"], rtol=1e-14)
    np.testing.assert_allclose(w, d[f"{tag}_w"], rtol=1e-14)
    p = unpack_params(d, "p_", O.Params)
    ev = unpack_events(d, "e_", O.Events)
    M = O.simulate_spread(p, ev, d["m0"], float(d["sigma_hz"]), shape, nodes)
    np.testing.assert_allclose(M, d[f"{tag}_M"], rtol=0, atol=1e-12)


def test_event_builders_match_the_reference():
    d = golden("events")
    ev = O.cw_saturation(np.linspace(-6, 6, 7), 1.5, 2.0, 3.0, m0_ppm=-300.0)
    for f in O.Events._fields:
        np.testing.assert_array_equal(np.asarray(getattr(ev, f), np.float64), np.asarray(d["cw_" + f], np.float64))
    st = O.stack_events([O.cw_saturation(np.linspace(-1, 1, 3), b, t, 2.8936) for b, t in ((0.5, 2.0), (1.0, 1.0))])
    for f in O.Events._fields:
        np.testing.assert_array_equal(np.asarray(getattr(st, f), np.float64), np.asarray(d["stack_" + f], np.float64))
    pd = O.pad_events(ev, 5)
    for f in O.Events._fields:
        np.testing.assert_array_equal(np.asarray(getattr(pd, f), np.float64), np.asarray(d["pad_" + f], np.float64))


def test_lm_on_rosenbrock_follows_the_reference():
    """fitting/lm.py on Rosenbrock (tests/test_fitting.py:90-100): same iterates, same end point."""
    d = golden("lm")

    def rj(x, need_jac=True):
        r = np.array([10.0 * (x[1] - x[0] ** 2), 1.0 - x[0]])
        J = np.array([[-20.0 * x[0], 10.0], [-1.0, 0.0]])
        return r, J
    x, X, C = O.levenberg_marquardt(rj, [-1.2, 1.0], [-5, -5], [5, 5], n_iter=200, trajectory=True)
    np.testing.assert_allclose(x, d["rosen_x"], atol=1e-9)
    np.testing.assert_allclose(C[:20], d["rosen_C"][:20], rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(X[:20], d["rosen_X"][:20], rtol=1e-6, atol=1e-9)


def test_oracle_jacobian_is_the_derivative_of_the_reference_model():
    """Exact forward mode (complex step + Frechet derivative) against central differences of the
    reference's own model (README ladder, k and f)."""
    d = golden("lm")
    s = golden("spectra")
    p = unpack_params(s, "readme_p_", O.Params)
    ev = unpack_events(s, "readme_e_", O.Events)
    k, f = d["jac_x"]
    q = p._replace(cest_k=np.array([k]), cest_f=np.array([f]))
    slots = [O.Slot("cest_k", 0), O.Slot("cest_f", 0)]
    sub = O.Events(*[np.asarray(a)[::8] for a in ev])             # every 8th offset: 31 chains
    Z, J = O.spectrum_jacobian(q, sub, s["readme_m0"], slots)
    np.testing.assert_allclose(J, d["jac_J"][::8], rtol=1e-4, atol=1e-8)   # central differences: ~1e-5


def test_readme_quick_start_fit_is_recovered():
    """README.md:62-94: the float64 reference fit of the 4-rung QUESP ladder returns the truth; the
    oracle LM from the same start reaches the same point. (The README's printed 49.617 / 9.0772e-4 is
    its float32 run, within 1% of this.)"""
    d = golden("lm")
    s = golden("spectra")
    p = unpack_params(s, "readme_p_", O.Params)
    ev = unpack_events(s, "readme_e_", O.Events)
    sub = O.Events(*[np.asarray(a)[::4] for a in ev])
    z = d["readme_z"][::4]
    slots = [O.Slot("cest_k", 0, 100.0), O.Slot("cest_f", 0, 0.001)]
    x = O.fit_voxel(p, sub, s["readme_m0"], slots, z, [300.0, 5e-4], [5.0, 1e-6], [5000.0, 0.05], n_iter=30)
    np.testing.assert_allclose(x, d["readme_x"][0], rtol=1e-5)
    np.testing.assert_allclose(d["readme_x"][0], [50.0, 9.009e-4], rtol=1e-6)
    assert abs(49.617 / x[0] - 1) < 0.01 and abs(9.0772e-4 / x[1] - 1) < 0.01


@pytest.mark.parametrize("tag", SPECTRA + ["quesp"])
def test_c_oracle_matches_the_reference(tag):
    """The compiled twin (oracle/bmc_oracle.c, Pade-13 scaling and squaring) on every golden case."""
    d = golden("spectra")
    p = unpack_params(d, f"{tag}_p_", O.Params)
    ev = unpack_events(d, f"{tag}_e_", O.Events)
    nc = O.n_cest_of(p)
    mz = int(d[f"{tag}_mz"])
    from bmc_b200.simulation import pack_params, SimParams
    z = O.c_simulate_z(pack_params(SimParams(*p), 1), ev, d[f"{tag}_m0"], nc, mz)
    np.testing.assert_allclose(z[0], d[f"{tag}_M"][:, mz], rtol=0, atol=1e-10)
