"""B200-native batched MAYO engine (keypair / sign / verify for MAYO_1/2/3/5).

The compute path is libmayo_b200.so (hand-written sm_100a CUDA behind a C-ABI, see
include/mayo_b200.h); this package is its host-side mirror of the reference API.
"""
from .api import A128, SETS, Mayo, MayoError, Sizes, aes128_tables_init, lib, sizes  # noqa: F401

__all__ = ["A128", "SETS", "Mayo", "MayoError", "Sizes", "aes128_tables_init", "lib", "sizes"]
