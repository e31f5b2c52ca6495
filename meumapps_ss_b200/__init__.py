"""B200-native (sm_100a) MEUMAPPS-SS time step behind a C-ABI.

``meumapps_ss_b200.sim.Simulation`` wraps the handle of ``include/meu.h``;
``params`` mirrors the reference's parameter set-up; ``configs`` builds decks.
"""
from . import params  # noqa: F401

__all__ = ["params"]
