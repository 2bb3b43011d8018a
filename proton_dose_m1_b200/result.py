"""Solver result container (proton_solver/result.py:10-153): same fields and
primary/reference selection, so code written against the reference's
``Result`` reads this one.  Plots and the reference's metric suite are not
part of this library; ``metrics`` gives this package's scoring functions
bound to the result."""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

from .enums import Backend


@dataclass
class Result:
    phi: Any
    J: Any
    dose: Any

    grid: Any
    energies: Any
    snapshots: dict[float, Any] = field(default_factory=dict)

    analytical_dose: Any = None
    topas_dose: Any = None
    bfp_mc_dose: Any = None

    runtime: float | None = None
    topas_runtime: float | None = None
    bfp_mc_runtime: float | None = None
    backend: Backend | None = None
    run_directory: Any = None

    x = property(lambda self: self.grid.x)
    y = property(lambda self: self.grid.y)
    z = property(lambda self: self.grid.z)

    def _mc_present(self):
        return self.bfp_mc_dose is not None or self.topas_dose is not None

    @property
    def primary_dose(self):
        """The deterministic dose when present, else BFP-MC, TOPAS, analytical."""
        for d in (self.dose, self.bfp_mc_dose, self.topas_dose, self.analytical_dose):
            if d is not None:
                return d
        return None

    @property
    def primary_label(self):
        for d, name in ((self.dose, "Deterministic"), (self.bfp_mc_dose, "BFP Monte Carlo"),
                        (self.topas_dose, "TOPAS"), (self.analytical_dose, "Analytical")):
            if d is not None:
                return name
        return None

    @property
    def reference_dose(self):
        """The comparison dose: analytical when a Monte Carlo result is itself
        the primary, else BFP-MC, TOPAS, analytical."""
        if self.dose is None and self.analytical_dose is not None and self._mc_present():
            return self.analytical_dose
        for d in (self.bfp_mc_dose, self.topas_dose, self.analytical_dose):
            if d is not None:
                return d
        return None

    @property
    def reference_label(self):
        if self.dose is None and self.analytical_dose is not None and self._mc_present():
            return "Analytical"
        for d, name in ((self.bfp_mc_dose, "BFP Monte Carlo"), (self.topas_dose, "TOPAS"),
                        (self.analytical_dose, "Analytical")):
            if d is not None:
                return name
        return None

    def compare(self, reference=None, gamma_cases=((1.0, 1.0),)):
        """Gamma, maximum dose, R80 and DFW of the primary dose against
        ``reference`` (default: the result's reference dose)."""
        from . import metrics
        ref = self.reference_dose if reference is None else reference
        if ref is None:
            raise ValueError("no reference dose to compare with")
        return metrics.compare(self.primary_dose, ref, self.grid, gamma_cases)
