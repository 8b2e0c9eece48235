"""The four example models BMC-JAX ships (io/configs/*.yaml), as plain objects with the attributes
`to_sim_params` reads (water_pool, cest_pools, mt_pool, system, options, mz_loc).

The YAML reader itself is outside this library's scope; these are the same numbers, rates given
as 1 / time where the YAML gives times.
"""
from dataclasses import dataclass, field
from typing import List, Optional

__all__ = ["Pool", "MTPool", "System", "Options", "Model", "example_config", "example_config_names"]


@dataclass(frozen=True)
class Pool:
    f: float
    r1: float
    r2: float
    k: float = 0.0
    dw: float = 0.0


@dataclass(frozen=True)
class MTPool(Pool):
    lineshape: str = "superlorentzian"


@dataclass(frozen=True)
class System:
    b0: float
    gamma: float = 267.5153
    b0_inhom: float = 0.0
    rel_b1: float = 1.0


@dataclass(frozen=True)
class Options:
    scale: float = 1.0
    max_pulse_samples: int = 200


@dataclass(frozen=True)
class Model:
    water_pool: Pool
    cest_pools: List[Pool] = field(default_factory=list)
    mt_pool: Optional[MTPool] = None
    system: System = System(3.0)
    options: Options = Options()

    @property
    def mz_loc(self) -> int:
        """Index of water Mz in the state vector (io/parameters/parameters.py:56-67)."""
        return 2 + 2 * len(self.cest_pools)

    @property
    def num_cest_pools(self) -> int:
        return len(self.cest_pools)


_WATER = Pool(f=1.0, r1=1 / 1.3, r2=1 / 0.05)
_AMIDE = Pool(f=0.0009009, r1=1 / 1.0, r2=1 / 0.1, k=50.0, dw=3.5)
_NOE = Pool(f=0.0045, r1=1 / 1.3, r2=1 / 0.005, k=20.0, dw=-3.0)
_MODELS = {
    "amide": Model(_WATER, [_AMIDE], None, System(3.0)),
    "amide_noe": Model(_WATER, [_AMIDE, _NOE], None, System(3.0)),
    "amide_noe_mt": Model(_WATER, [_AMIDE, _NOE],
                          MTPool(f=0.05, r1=1.0, r2=1 / 1.0e-05, k=30.0, dw=-2.5, lineshape="superlorentzian"),
                          System(3.0)),
    "phantom_creatine": Model(Pool(f=1.0, r1=0.3039, r2=0.613), [Pool(f=0.00324, r1=1.0, r2=33.3, k=104.5, dw=1.9)],
                              None, System(2.8936, 267.5153, -0.07, 1.027)),
}


def example_config_names():
    return sorted(_MODELS)


def example_config(name: str) -> Model:
    """One of the shipped example models by name (io/config.py)."""
    try:
        return _MODELS[name]
    except KeyError:
        raise ValueError(f"no example config {name!r}; choose from {example_config_names()}") from None
