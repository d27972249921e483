"""B200-native IFGF matvec (Interpolated Factored Green Function).

A from-scratch CUDA (sm_100a) implementation of the matvec of TimHRO/ifgf's
IfgfOperator with its six kernel plug-ins, behind a C ABI
(include/ifgf_b200.h, libifgf_b200.so) and the reference's Python operator
API (``ifgf_b200.pyifgf`` carries the reference module's names).
"""
from ._lib import IfgfError  # noqa: F401  (fails loudly if the CUDA library is missing)
from .operators import (  # noqa: F401
    CombinedFieldHelmholtzIfgfOperator,
    DoubleLayerHelmholtzIfgfOperator,
    GradHelmholtzIfgfOperator,
    HelmholtzIfgfOperator,
    IfgfOperator,
    LaplaceIfgfOperator,
    ModifiedHelmholtzIfgfOperator,
    MofifiedHelmholtzIfgfOperator,
)

__version__ = "0.1.0"
