"""B200-native CabanaPD hot path: peridynamics (PMB, LPS) and Hertzian DEM
particle kernels in hand-written sm_100a CUDA behind a C ABI."""
from .inputs import Inputs, critical_timestep  # noqa: F401
from . import problems  # noqa: F401
from .system import System, Server, Batch, CpdError, load as load_library  # noqa: F401
