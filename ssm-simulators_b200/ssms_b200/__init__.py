"""ssms_b200 -- sm_100a (B200) implementation of ssm-simulators' hot path.

Drop-in surfaces:
  * ``ssms_b200.cssm``      -- the reference's ``cssm`` simulator entry points
  * ``ssms_b200.Simulator`` -- ``Simulator(model).simulate(theta, n_samples)``
  * ``ssms_b200.device``    -- the same simulators on CUDA tensors (no host copies)

All simulation runs in ``libssm_b200.so`` (hand-written CUDA for sm_100a),
called through a C ABI (include/ssm_b200.h) with ctypes.
"""

from . import boundary_functions, cssm  # noqa: F401
from .config import ModelConfigBuilder, model_config  # noqa: F401
from .simulator import OMISSION_SENTINEL, Simulator, simulator  # noqa: F401

__version__ = "0.1.0"
