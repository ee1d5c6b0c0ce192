"""gpuequiv_b200 - B200-native solver for the energy games of gpuequiv.

The package mirrors the public API of the gpuequiv crate (EnergyConf, Energy,
EnergyArray, Upd/Update/UpdateArray, GameGraph, EnergyGame, GameBuild,
TransitionSystem, Equivalence) over the C ABI of ``libgeq.so``
(``include/geq.h``), whose CUDA kernels for sm_100a solve the games.
"""
from ._lib import GeqError, library_path
from .energy import (Energy, EnergyArray, EnergyConf, Upd, Update, UpdateArray, std_equivalences,
                     update)
from .energygame import (Context, DeviceGames, EnergyGame, GameGraph, b_min, c_views, default_context, run_batch,
                         run_batch_raw, run_static)
from .lts import (Equivalence, EquivalenceRelation, GameBatch, GameBuild, Position, StartInfo,
                  TransitionSystem, compare_batch, signature_refinement_batch)

__all__ = [
    "GeqError", "library_path", "Energy", "EnergyArray", "EnergyConf", "Upd", "Update", "UpdateArray",
    "std_equivalences", "update", "Context", "DeviceGames", "EnergyGame", "GameGraph", "default_context",
    "run_batch", "run_batch_raw", "run_static", "c_views", "b_min", "Equivalence", "EquivalenceRelation", "GameBatch", "GameBuild", "Position", "StartInfo",
    "TransitionSystem", "compare_batch", "signature_refinement_batch",
]
