"""Drop-in for the reference's ``pyifgf`` module (py_ifgf.cpp:25-58).

``from ifgf_b200 import pyifgf`` (or putting this package's ``pyifgf`` on the
import path as ``pyifgf``) gives the three classes the reference binds, with
the same names, constructor arguments, ``init`` and ``mult``.  The reference
binds the modified Helmholtz operator under a misspelled name
(``MofifiedHelmholtzIfgfOperator``, py_ifgf.cpp:37-38); both that name and
the correct spelling refer to the same class here.
"""
from .operators import (  # noqa: F401
    GradHelmholtzIfgfOperator,
    LaplaceIfgfOperator,
    ModifiedHelmholtzIfgfOperator,
    MofifiedHelmholtzIfgfOperator,
)

__version__ = "dev"  # py_ifgf.cpp:55-57
