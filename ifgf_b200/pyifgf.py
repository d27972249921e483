"""Drop-in for the reference's ``pyifgf`` module (py_ifgf.cpp:25-58).

``from ifgf_b200 import pyifgf`` (or putting this package's ``pyifgf`` on the
import path as ``pyifgf``) gives the three classes the reference binds, with
the same names, constructor arguments, ``init`` and ``mult``.
"""
from .operators import (  # noqa: F401
    GradHelmholtzIfgfOperator,
    LaplaceIfgfOperator,
    MofifiedHelmholtzIfgfOperator,
)

__version__ = "dev"  # py_ifgf.cpp:55-57
