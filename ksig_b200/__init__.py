"""ksig_b200: B200 (sm_100a) signature kernels with KSig's callable API.

Importing the package does not touch the GPU; the CUDA library
(``lib/libksig_b200.so``) is loaded on first use.
"""

from . import graphs  # noqa: F401
from . import kernels  # noqa: F401
from . import precompute  # noqa: F401
from . import preprocessing  # noqa: F401
from . import static  # noqa: F401
from . import tuning  # noqa: F401
from . import utils  # noqa: F401
from .graphs import GraphedKernel  # noqa: F401
from .kernels import (GlobalAlignmentKernel, Ragged, SignatureKernel,  # noqa: F401
                      SignaturePDEKernel)
from .static.kernels import (LinearKernel, Matern12Kernel, Matern32Kernel,  # noqa: F401
                             Matern52Kernel, PolynomialKernel, RationalQuadraticKernel,
                             RBFKernel)

from ._engine import check_device_status  # noqa: F401

__version__ = '0.1.0'
