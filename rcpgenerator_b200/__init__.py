"""rcpgenerator_b200: RCPGenerator's packing engine on one NVIDIA B200.

Drop-in for the relaxation path of RCPGenerator (``Packing(...).pack()``):
the same ``Packing`` class and the same module functions as the reference
package ``rcpgenerator`` / its binding ``_rcpgenerator``, computed by
hand-written sm_100a CUDA kernels behind a C ABI (include/rcpg.h).

Submodules: ``warmstart`` (the learned warm start: network, training,
evaluation), ``jobs`` (the rcptools job loop on the batch engine and the GPU
overlap report), ``train_warmstart`` (command-line trainer).
"""

from ._api import (
    PackingEngine,
    batch_tuning,
    get_num_threads,
    initialize_particles,
    run_packing,
    run_packing_batch,
    run_packing_observed,
    set_num_threads,
)
from ._wrapper import Packing

__all__ = [
    "Packing",
    "PackingEngine",
    "batch_tuning",
    "get_num_threads",
    "initialize_particles",
    "run_packing",
    "run_packing_batch",
    "run_packing_observed",
    "set_num_threads",
]
