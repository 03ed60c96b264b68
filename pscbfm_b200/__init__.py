"""B200-native engine for the parallel Monte Carlo sweep of the simple-cubic bond fluctuation
model: a drop-in for pscbfm's UpdaterGPUScBFM_AB_Type.

The product is the C-ABI library libbfm.so (include/bfm.h, sources in csrc/); this package is
its Python host binding (updater.py), the synthetic systems it is measured on (systems.py) and
the build script (build.py).
"""
from .updater import UpdaterGPUScBFM_AB_Type, Batch, MODE_AUTO, MODE_LAUNCH, MODE_GRAPH, MODE_RESIDENT  # noqa: F401
from .updater import MODE_PERSISTENT, MODE_CLUSTER  # noqa: F401
from .updater import REPR_AUTO, REPR_GATHER, Server, probe_device  # noqa: F401
from ._lib import BfmCudaError, BfmBudgetError, BfmBusy  # noqa: F401
from .sharding import shard_systems, run_sharded, batch_runner  # noqa: F401
