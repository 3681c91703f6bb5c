"""B200-native Coulomb-integral path (McMurchie-Davidson) with the reference's C ABI.

Import with ``importlib.import_module("electron-integral-playground_b200")``
(the directory name is not a Python identifier).
"""

from .data_structure import GaussianShell, Molecule, PrimitivePairData  # noqa: F401
