"""Generate the golden vectors in this folder by EXECUTING THE REFERENCE'S OWN SOURCE.

Run where the BMC-JAX source tree is available, passing its `src` folder:

    python tests/golden/make_golden.py /path/to/BMC-JAX/src

JAX is not installable here, so `_jaxshim/jax` stands in for the JAX API subset the reference uses,
eagerly and in float64 (see its docstring). Everything below calls reference functions by their
public names -- bmc_matrix, simulate_spectrum, simulate_spectrum_spread, cw_saturation,
Experiment.stack, pad_events, levenberg_marquardt, fit -- and saves inputs and outputs. Events are
cast to float64 with the reference's `cast_events` so that the whole computation is float64 (its
`cw_saturation` emits float32 events, which under JAX's weak typing would keep 2*pi*rf_freq and
cos(rf_phase) in float32).

Jacobians: the stand-in's jacfwd is a central difference, so `jac_*` fixtures are the reference's
model differentiated numerically (accurate to ~1e-5 relative: the 2 s CW steps carry ~1e-13 of
rounding); the exact forward-mode Jacobians of the oracle and of the CUDA path are checked against
them at 1e-4, and against each other far more tightly.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py /path/to/BMC-JAX/src")
REF_SRC = sys.argv[1]
sys.path.insert(0, str(HERE / "_jaxshim"))
sys.path.insert(0, REF_SRC)

import jax                                                      # noqa: E402  (the stand-in)
import jax.numpy as jnp                                         # noqa: E402
from bmc_jax.io import example_config                           # noqa: E402
from bmc_jax.simulation import (to_sim_params, initial_state, simulate_spectrum, bmc_matrix,   # noqa: E402
                                cast_events, pad_events, B0Spread, simulate_spectrum_spread,
                                SimEvent, EventType)
from bmc_jax.sequences import cw_saturation                     # noqa: E402
from bmc_jax.fitting import Experiment, FitSpec, FreeParam, fit, levenberg_marquardt   # noqa: E402

F64 = np.float64
PFIELDS = ("water_r1", "water_r2", "water_f", "cest_k", "cest_f", "cest_dw", "cest_r1", "cest_r2",
           "mt_k", "mt_f", "mt_dw", "mt_r1", "mt_r2", "mt_lineshape", "b0", "gamma", "b0_inhom", "rel_b1")
EFIELDS = ("type", "dt", "rf_amp", "rf_phase", "rf_freq", "adc_idx")


def pack_params(jp, prefix="p_"):
    return {prefix + f: np.asarray(getattr(jp, f)) for f in PFIELDS}


def pack_events(ev, prefix="e_"):
    return {prefix + f: np.asarray(getattr(ev, f)) for f in EFIELDS}


def spectrum(jp, ev, m0):
    return np.asarray(simulate_spectrum(jp, ev, m0, return_full_trajectory=False))


def ev64(ev):
    return cast_events(ev, F64)


def main():
    out = {}

    # 1. system matrices for every lineshape branch and RF state ------------------------------
    mats = {}
    cases = [("amide", 10.0, 0.3, 100.0), ("amide_noe", 42.0, 1.0, -300.0),
             ("amide_noe_mt", 5.0, 0.0, -900.0), ("amide_noe_mt", 25.0, 2.0, -290.0),
             ("amide_noe_mt", 25.0, -1.0, 40.0), ("phantom_creatine", 12.0, 0.7, 250.0)]
    for i, (name, a, ph, fr) in enumerate(cases):
        jp = to_sim_params(example_config(name))
        if i == 4:                              # Lorentzian MT lineshape
            jp = jp._replace(mt_lineshape=np.asarray(1))
        A, C = bmc_matrix(jp, a, ph, fr)
        mats.update({f"m{i}_A": np.asarray(A), f"m{i}_C": np.asarray(C), f"m{i}_rf": np.array([a, ph, fr])})
        mats.update(pack_params(jp, f"m{i}_p_"))
    np.savez_compressed(HERE / "matrix.npz", **mats)

    # 2. spectra --------------------------------------------------------------------------------
    spec = {}

    def add(tag, jp, ev, m0, mz):
        z = spectrum(jp, ev, m0)
        spec.update(pack_params(jp, f"{tag}_p_"))
        spec.update(pack_events(ev, f"{tag}_e_"))
        spec[f"{tag}_m0"] = np.asarray(m0)
        spec[f"{tag}_mz"] = np.asarray(mz)
        spec[f"{tag}_M"] = z

    # README quick-start: amide, QUESP ladder 0.5/1/2/4 uT, 2 s CW, 61 offsets (README.md:62-94)
    p = example_config("amide")
    jp = to_sim_params(p)
    m0 = initial_state(jp)
    ppm = np.linspace(-6, 6, 61)
    ladder = Experiment.stack([Experiment(jp, ev64(cw_saturation(ppm, b, 2.0, p.system.b0)), m0, p.mz_loc)
                               for b in (0.5, 1.0, 2.0, 4.0)])
    add("readme", jp, ladder.events, m0, p.mz_loc)

    # MT pool, super-Lorentzian (both branches) and Lorentzian; CW at 1.5 uT
    p = example_config("amide_noe_mt")
    jp = to_sim_params(p)
    ev = ev64(cw_saturation(np.linspace(-6, 6, 49), 1.5, 1.0, p.system.b0))
    add("mt_sl", jp, ev, initial_state(jp, 0.8), p.mz_loc)
    add("mt_lor", jp._replace(mt_lineshape=np.asarray(1)), ev, initial_state(jp), p.mz_loc)

    # field and amplitude calibration off nominal
    p = example_config("phantom_creatine")
    jp = to_sim_params(p)
    add("creatine", jp, ev64(cw_saturation(np.linspace(-4, 4, 33), 0.8, 3.0, p.system.b0, m0_ppm=-300.0)),
        initial_state(jp, 0.557), p.mz_loc)

    # shipped pulsed QUESP train (4041 events: recovery, 20 x (200 RF samples, spoiler, gap), spoiler, ADC)
    d = np.load(Path(REF_SRC).parent / "examples" / "data" / "events" / "quesp_sim_b1_1uT_events.npz")
    rows = [0, 1, 26, 51, 60, 101]
    ev = SimEvent(*[np.asarray(d[f][rows]).astype(np.int32 if f in ("type", "adc_idx") else F64) for f in EFIELDS])
    add("quesp", jp, ev, initial_state(jp, 0.557), p.mz_loc)

    # event semantics: GRADIENT spoils like SPOILER, an ADC with a duration evolves, events after an
    # ADC start from the reset state, zero-length events of every type are no-ops
    jp = to_sim_params(example_config("amide_noe"))
    T = [EventType.DELAY, EventType.RF_PULSE, EventType.GRADIENT, EventType.RF_PULSE, EventType.ADC,
         EventType.RF_PULSE, EventType.SPOILER, EventType.RF_PULSE, EventType.ADC, EventType.RF_PULSE,
         EventType.RF_PULSE, EventType.DELAY]
    DT = [0.5, 0.02, 0.001, 0.3, 0.004, 0.01, 0.0, 0.05, 0.0, 1e-10, 0.003, 0.2]
    AMP = [0.0, 80.0, 0.0, 30.0, 0.0, 50.0, 10.0, 40.0, 0.0, 500.0, 60.0, 0.0]
    PH = [0.0, 0.4, 0.0, -1.2, 0.0, 2.0, 0.0, 0.1, 0.0, 0.0, 3.0, 0.0]
    n_off = 5
    fr = np.linspace(-700.0, 500.0, n_off)[:, None] * np.ones(len(T))
    ev = SimEvent(type=np.tile(np.int32(T), (n_off, 1)), dt=np.tile(F64(DT), (n_off, 1)),
                  rf_amp=np.tile(F64(AMP), (n_off, 1)), rf_phase=np.tile(F64(PH), (n_off, 1)),
                  rf_freq=fr.astype(F64), adc_idx=np.tile(np.int32([-1] * 4 + [0] + [-1] * 3 + [1, -1, -1, -1]), (n_off, 1)))
    add("semantics", jp._replace(b0_inhom=np.asarray(0.05), rel_b1=np.asarray(0.9)), ev, initial_state(jp, 0.7), 6)

    # front padding (bit-exact no-op) and the tail-padding trap (returns the start state)
    p = example_config("amide")
    jp = to_sim_params(p)
    ev = ev64(cw_saturation(np.linspace(-5, 5, 21), 1.0, 2.0, p.system.b0))
    add("front_pad", jp, pad_events(ev, ev.dt.shape[1] + 37), initial_state(jp), p.mz_loc)
    tail = SimEvent(*[np.concatenate([np.asarray(getattr(ev, f)),
                                      np.full((21, 4), {"type": 0, "adc_idx": -1}.get(f, 0.0),
                                              np.asarray(getattr(ev, f)).dtype)], axis=1) for f in EFIELDS])
    add("tail_pad", jp, tail, initial_state(jp), p.mz_loc)
    np.savez_compressed(HERE / "spectra.npz", **spec)

    # 3. B0 spread ------------------------------------------------------------------------------
    sp = {}
    p = example_config("amide")
    jp = to_sim_params(p)
    ev = ev64(cw_saturation(np.linspace(-3, 3, 25), 1.0, 1.0, p.system.b0))
    m0 = initial_state(jp)
    for tag, s in (("gauss5", B0Spread(shape="gauss", nodes=5)), ("lorentz3", B0Spread(shape="lorentz", nodes=3, cut=20.0))):
        z = np.asarray(simulate_spectrum_spread(jp, ev, m0, 12.0, s))
        u, w = s.nodes_weights()
        sp.update({f"{tag}_M": z, f"{tag}_u": u, f"{tag}_w": w})
    sp.update(pack_params(jp))
    sp.update(pack_events(ev))
    sp["m0"] = np.asarray(m0)
    sp["sigma_hz"] = np.asarray(12.0)
    np.savez_compressed(HERE / "spread.npz", **sp)

    # 4. event builders -------------------------------------------------------------------------
    ev = cw_saturation(np.linspace(-6, 6, 7), 1.5, 2.0, 3.0, m0_ppm=-300.0)
    stk = Experiment.stack([Experiment(None, cw_saturation(np.linspace(-1, 1, 3), b, t, 2.8936), None, 4)
                            for b, t in ((0.5, 2.0), (1.0, 1.0))])
    padded = pad_events(ev, 5)
    builders = {**pack_events(ev, "cw_"), **pack_events(stk.events, "stack_"), **pack_events(padded, "pad_")}
    np.savez_compressed(HERE / "events.npz", **builders)

    # 5. LM without physics (tests/test_fitting.py:90-100) and the README fit ---------------------
    lm = {}

    def rosen(x):
        return jnp.array([10.0 * (x[1] - x[0] ** 2), 1.0 - x[0]])
    x, X, C = levenberg_marquardt(rosen, jnp.array([-1.2, 1.0]), jnp.array([-5.0, -5.0]), jnp.array([5.0, 5.0]),
                                  n_iter=200, return_trajectory=True)
    lm.update(rosen_x=np.asarray(x), rosen_X=np.asarray(X), rosen_C=np.asarray(C))

    p = example_config("amide")
    jp = to_sim_params(p)
    m0 = initial_state(jp)
    ppm = np.linspace(-6, 6, 61)
    ladder = Experiment.stack([Experiment(jp, ev64(cw_saturation(ppm, b, 2.0, p.system.b0)), m0, p.mz_loc)
                               for b in (0.5, 1.0, 2.0, 4.0)])
    z = np.asarray(ladder.simulate())
    spec_ = FitSpec([FreeParam("k", "cest_k", 0, scale=100.0, lo=5.0, hi=5000.0, x0=300.0),
                     FreeParam("f", "cest_f", 0, scale=0.001, lo=1e-6, hi=0.05, x0=0.0005)])
    res = fit(ladder, spec_, z[None, :], n_per_block=len(ppm))
    lm.update(readme_x=np.asarray(res.x), readme_z=z, readme_zfit=np.asarray(res.z_fit))

    # Jacobian of the README model at (k, f) = (120, 6e-4), central differences on the reference
    def model(x):
        q = jp._replace(cest_k=jnp.asarray([x[0]]), cest_f=jnp.asarray([x[1]]))
        return np.asarray(simulate_spectrum(q, ladder.events, m0, return_full_trajectory=False))[:, p.mz_loc]
    x0 = np.array([120.0, 6e-4])
    J = np.empty((z.size, 2))
    for j, h in enumerate((1e-3, 2e-8)):
        e = np.zeros(2); e[j] = h
        J[:, j] = (model(x0 + e) - model(x0 - e)) / (2 * h)
    lm.update(jac_x=x0, jac_J=J)
    np.savez_compressed(HERE / "lm.npz", **lm)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
