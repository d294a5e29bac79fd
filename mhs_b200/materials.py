"""The elastic material as ``(mu, lam)`` -- the value type every matrix call
takes, with mhs's admissibility rules (mhs/materials.py:33-84)."""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Material:
    """Isotropic linear elastic material: shear modulus ``mu`` and Lame's
    first parameter ``lam``.  Coefficients are formed from ``(mu, lam)``; no
    ``1 / (1 - 2 nu)`` is ever taken."""

    mu: float
    lam: float

    def __post_init__(self) -> None:
        if not (self.mu > 0.0):
            raise ValueError(f"mu must be positive, got {self.mu!r}")
        if not (self.lam > -2.0 * self.mu / 3.0):
            raise ValueError(
                f"lam must exceed -2 mu / 3 = {-2.0 * self.mu / 3.0!r} for a "
                f"positive bulk modulus, got {self.lam!r}")

    @property
    def bulk(self) -> float:
        """``K = lam + 2 mu / 3``."""
        return self.lam + 2.0 * self.mu / 3.0

    @property
    def nu_if_you_must(self) -> float:
        """Poisson's ratio, for code that insists on it."""
        return 0.5 * self.lam / (self.lam + self.mu)

    @classmethod
    def from_mu_nu(cls, mu: float, nu: float) -> "Material":
        """Build from ``(mu, nu)``; refuses ``nu >= 1/2``."""
        if not (-1.0 < nu < 0.5):
            raise ValueError(
                f"nu must lie in (-1, 1/2) to convert to lam; got {nu!r}. "
                f"An incompressible material has no finite lam -- construct "
                f"Material(mu, lam) with a large lam directly.")
        return cls(mu=float(mu), lam=2.0 * float(mu) * nu / (1.0 - 2.0 * nu))
