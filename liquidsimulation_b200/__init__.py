"""liquidsimulation_b200: LiquidPhysics' SPH / PCISPH particle step on B200 (sm_100a)."""
from . import abi, scenes  # noqa: F401

__all__ = ["abi", "scenes"]
