"""fenice_b200: the uniform-grid finite-volume right-hand side and time step of the Fenice solver, rebuilt for the
NVIDIA B200 (sm_100a): hand-written CUDA kernels behind a C ABI (include/fenice_gpu.h), with this package as the Python
host binding. See ``fenice_b200.runtime.Run``."""
from .params import load_case, resolve, to_config  # noqa: F401
from .runtime import Batch, BatchProblem, Run, StepResult, load_library  # noqa: F401
