"""The 3D step: containers (:mod:`.types`), set-up (:mod:`.setup`), the C-ABI plan
(:mod:`.plan`), the reference-facing drop-in (:mod:`.fused`) and workloads."""
from .types import DyeSources, Geometry3D, Ops3D, State3D, StepOut3D, ThermalGeometry, ThermalOps

__all__ = ["DyeSources", "Geometry3D", "Ops3D", "State3D", "StepOut3D", "ThermalGeometry", "ThermalOps"]
