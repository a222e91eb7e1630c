"""fresco_b200: B200-native loss-and-gradient path of FReSCo.

``fresco_b200.potentials`` and ``fresco_b200.optimize`` mirror the reference's
``fresco.potentials`` and ``fresco.optimize``.  ``install_alias()`` registers
them under the reference's import names so existing scripts run unchanged::

    import fresco_b200
    fresco_b200.install_alias()
    from fresco.potentials import NUwU
    from fresco.optimize import LBFGS_CPP
"""
from __future__ import annotations

import sys
import types

from . import _lib  # noqa: F401  (loads the CUDA library; raises ImportError if missing)
from . import distances, ensemble, optimize, potentials, shard, utils
from .ensemble import EnsembleLBFGS, NUwUEnsemble
from .potentials import CombinedPotential, InversePower, NUwNU, NUwU, UwNU, UwU
from .shard import ShardedLBFGS, ShardedNUwU

__all__ = ["potentials", "optimize", "utils", "distances", "ensemble", "shard", "install_alias", "NUwU", "UwU", "UwNU", "NUwNU",
           "InversePower", "CombinedPotential", "NUwUEnsemble", "EnsembleLBFGS", "ShardedNUwU", "ShardedLBFGS"]


def install_alias() -> None:
    """Makes ``import fresco.potentials`` / ``fresco.optimize`` / ``fresco.utils`` / ``fresco.distances`` resolve
    to this package."""
    pkg = types.ModuleType("fresco")
    pkg.__path__ = []  # namespace-like
    pkg.potentials = potentials
    pkg.optimize = optimize
    pkg.utils = utils
    pkg.distances = distances
    sys.modules.setdefault("fresco", pkg)
    sys.modules.setdefault("fresco.potentials", potentials)
    sys.modules.setdefault("fresco.optimize", optimize)
    sys.modules.setdefault("fresco.utils", utils)
    sys.modules.setdefault("fresco.distances", distances)
