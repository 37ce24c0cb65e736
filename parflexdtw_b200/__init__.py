"""parflexdtw_b200 -- ParFlex (sparse parallel FlexDTW) alignment on NVIDIA B200.

The public functions keep the reference's (ishitajain21/ParFlexDTW) API:
``parflex``, ``tiled_stage1_from_features``, ``run_stage2_from_tiled``,
``run_flexdtw_on_tiles`` and ``flexdtw_chunk_from_global_C``; ``parflex_batch``
aligns many pairs of uneven lengths in one device batch.  They run on
hand-written sm_100a CUDA kernels behind the C ABI in
``include/parflexdtw_b200.h``; there is no CPU path.
"""
from .batch import Batch, parflex_batch  # noqa: F401
from .prune import PrunedBatch, TileProposer, parflex_pruned  # noqa: F401
from .parflex import (  # noqa: F401
    DEFAULT_CHUNK_LENGTH,
    ChunksDict,
    Plan,
    Stage2Result,
    TiledResult,
    buffer_global,
    clear_plan_cache,
    cost_matrix_from_features_gpu,
    cost_matrix_to_gpu,
    cost_matrix_to_gpu_f32,
    flexdtw,
    flexdtw_chunk_from_global_C,
    is_gpu_available,
    parflex,
    run_flexdtw_on_tiles,
    run_stage2_from_tiled,
    tiled_stage1_from_features,
)

__version__ = "0.1.0"
