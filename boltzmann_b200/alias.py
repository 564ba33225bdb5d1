"""Import aliases for code written against the reference's Python package.

``install()`` registers this backend under the reference's module names, so that scripts and
tests written for djbarker/boltzmann run on the CUDA backend without edits:

    ``boltzmann``             -> ``boltzmann_b200``
    ``boltzmann.boltzmann``   -> ``boltzmann_b200.boltzmann`` (the compiled classes, src/lib.rs)
    ``boltzmann.core``        -> ``boltzmann_b200.core`` (python/boltzmann/core.py)
    ``boltzmann.simulation``  -> ``boltzmann_b200.driver`` (run_sim and its gaters,
                                 python/boltzmann/simulation.py:31-271)

    import boltzmann_b200.alias
    boltzmann_b200.alias.install()
    from boltzmann.core import Simulation, bgk     # the CUDA backend

Modules of the reference outside the hot path (units, utils, mock, kernel_gen) are not aliased.
A ``boltzmann`` package that is already imported is left alone unless ``force`` is set.
"""

from __future__ import annotations

import importlib
import sys

ALIASES = {
    "boltzmann": "boltzmann_b200",
    "boltzmann.boltzmann": "boltzmann_b200.boltzmann",
    "boltzmann.core": "boltzmann_b200.core",
    "boltzmann.simulation": "boltzmann_b200.driver",
}


def install(force: bool = False) -> None:
    """Makes ``import boltzmann...`` resolve to this package's modules."""
    if "boltzmann" in sys.modules and not force:
        if sys.modules["boltzmann"] is importlib.import_module("boltzmann_b200"):
            return
        raise ImportError("a different 'boltzmann' package is already imported")
    for alias, target in ALIASES.items():
        sys.modules[alias] = importlib.import_module(target)
    parent = sys.modules["boltzmann"]
    for alias in ALIASES:
        if "." in alias:
            # attribute access (boltzmann.core) as after a normal submodule import; the package
            # object is boltzmann_b200 itself, so only names it lacks are added
            name = alias.split(".", 1)[1]
            if not hasattr(parent, name) or force:
                setattr(parent, name, sys.modules[alias])
