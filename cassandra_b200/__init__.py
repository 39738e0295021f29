"""cassandra_b200 — B200-native pattern-evaluator fitting path.

Positions -> ternary pattern indices (bit-exact with the reference's
GroupIndexer) -> device CSR + sort-built transposed copy -> Jacobi-PCG / LSQR
in plain FP64 or mixed precision, all as hand-written sm_100a CUDA kernels
behind the C ABI in include/cassandra_b200.h.
"""
from ._lib import CasError, SizeMismatch, load  # noqa: F401
from .api import (  # noqa: F401
    CG,
    DEFAULT_ACCURACY,
    LSMR,
    LSQR,
    PCG,
    GroupIndexer,
    MatrixCSR,
    MultiStageScoreEstimator,
    estimator_stages,
    fit_weights,
    fit_weights_batched,
    generate_positions,
    generate_positions_host,
    generate_targets,
    jacobi_preconditioner_of_ata,
    load_estimator,
    read_records,
    read_scored_positions,
    save_estimator,
    solve_batched,
    solve_opts,
)

# The 5- and 8-pattern sets of the fitting workloads (repo bit order, bit 0 = H8):
# edge+2X, 3x3 corner, 2x5 corner, main diagonal, row 2; then rows 3 and 4 and
# the 7-square diagonal.
PATTERNS_5 = [0x42FF, 0x070707, 0x1F1F, 0x8040201008040201, 0xFF00]
PATTERNS_8 = PATTERNS_5 + [0xFF0000, 0xFF000000, 0x0080402010080402]
