"""B200 density-fitting Coulomb/exchange backend for dftax.

The compute path is ``libdfjk.so`` (CUDA, sm_100a) behind the C ABI of
``include/dfjk.h``; this package holds its Python bindings, the host mirror of
dftax's Coulomb-backend interface, the closed-shell Kohn-Sham model and SCF
(``include/dfscf.h``), the Becke grid and the basis layout helpers.
"""

from .basis import BasisData, build_basis_data, cart2sph_block  # noqa: F401
from .coulomb import (B200DFCoulomb, Context, CoulombTerm, DFSpec, Plan, df,  # noqa: F401
                      make_coulomb)
from .grid import Becke, becke, becke_grid  # noqa: F401
from .ks import KS, KSResult, scf  # noqa: F401

__all__ = ["BasisData", "build_basis_data", "cart2sph_block", "B200DFCoulomb", "Context",
           "CoulombTerm", "DFSpec", "Plan", "df", "make_coulomb", "Becke", "becke", "becke_grid",
           "KS", "KSResult", "scf"]
