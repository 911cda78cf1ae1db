"""ugb200 -- B200-native RSA worldline packer (host side).

The compute path is libug.so (hand-written sm_100a CUDA behind the C ABI of
include/ug.h); this package is its Python host side: configuration, the
batch runner, result readers, the braid_cuda-compatible command line
(``python -m ugb200.cli``) and the dump / curve writers.
"""

from ._lib import (  # noqa: F401
    EXCL_OPEN, EXCL_REF, GROUP_NONE, GROUP_SUBPATH, GROUP_UNIQUE, PREC_FP64, PREC_MIXED,
    RNG_KNOT, RNG_PHILOX, ZGRID_MID, ZGRID_REF, UgError, load,
)
from .packer import Packer, Stats, Universe, load_checkpoint, pack, save_checkpoint  # noqa: F401
