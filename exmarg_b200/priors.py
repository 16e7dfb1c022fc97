"""Distance priors of the analysis (the contract of exmarg/priors.py:31-38).

'volume' is integrated in closed form (density None); 'madau-dickinson' is the
density of ln y tabulated in exmarg's package data (data/demo_population.npz,
members lny and p_lny), read from the installed exmarg package without importing
it.  A (lny, p_lny) pair can also be passed directly.
"""

import importlib.util
import os

import numpy as np


def _population_file():
    spec = importlib.util.find_spec("exmarg")
    if spec is None or not spec.submodule_search_locations:
        return None
    for loc in spec.submodule_search_locations:
        f = os.path.join(loc, "data", "demo_population.npz")
        if os.path.exists(f):
            return f
    return None


def distance_density(prior):
    if isinstance(prior, (tuple, list)) and len(prior) == 2:
        return np.asarray(prior[0], float), np.asarray(prior[1], float)
    if prior == "volume":
        return None
    if prior == "madau-dickinson":
        f = _population_file()
        if f is None:
            raise FileNotFoundError("the 'madau-dickinson' prior needs exmarg's data/demo_population.npz "
                                    "(install exmarg, or pass (lny, p_lny))")
        z = np.load(f)
        return np.asarray(z["lny"], float), np.asarray(z["p_lny"], float)
    raise ValueError("the distance prior is 'volume' or 'madau-dickinson', not %r" % (prior,))
