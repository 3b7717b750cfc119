"""The names the reference's system/tmine/core.py imports from corelib."""
import os
import sys

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from corelib import (  # noqa: E402,F401
    GPUWorker, GPUWorkerLibManager, MultiGPUExecutionDyn, MultiGPUExecutionDynPause,
    MultiGPUExecutionNaive, SingleGPUExecution, SingleGPUExecutionDiv, SingleGPUExecutionPause,
    SingleGPURunBatch, allCount, data,
)
import corelib  # noqa: E402,F401
