"""Field-circuit coupling: a meshed field region as a netlist element."""

from .coupling import FieldCircuitSystem, FieldRegion

__all__ = ["FieldRegion", "FieldCircuitSystem"]
