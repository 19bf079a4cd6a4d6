"""adgpu_b200: a B200-native engine for AutoDock-GPU's LGA docking hot path.

Modules: abi (C layout types), lib (the shared library), frontend (grid maps
and ligand preparation), device (reference kernel API plumbing), dock (plain
per-ligand docking), engine (batch / serving engine), synth (seeded synthetic
inputs).  device and dock need torch; the rest do not.
"""
from . import abi, lib, frontend, engine, result  # noqa: F401

__all__ = ["abi", "lib", "frontend", "engine"]
