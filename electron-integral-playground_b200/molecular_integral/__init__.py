"""Integral entry points with the reference front end's names and semantics
(electron_integral_playground/molecular_integral/*.py): one C call per
angular class, outputs zero-filled here and accumulated by the library."""

from .nuclear_attraction import nuclear_attraction  # noqa: F401
from .overlap import overlap  # noqa: F401
from .three_center import three_center  # noqa: F401
from .two_center import two_center  # noqa: F401
