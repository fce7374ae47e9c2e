"""B200-native (sm_100a) NRG step core: batched FP64 block diagonalisation, recalculation
of irreducible matrix elements and DM-NRG/FDM spectral-weight binning, behind a C-ABI
(include/nrg_b200.h) with a host mirror of NRG Ljubljana's interfaces (api.py)."""
from ._lib import NRGError, load as load_library  # noqa: F401
from .api import (BinGrid, Context, RawEigen, context, diag_batch_device, diagonalisations,  # noqa: F401
                  diagonalise, gemm3, gemm3_batch, is_matrix_upper, product, rotate, spec_accumulate, spec_pair,
                  transform)
