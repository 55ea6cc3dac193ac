"""B200-native Brownian-dynamics step for BD_BOX decks.

The product is the C-ABI library ``bd_box_b200/libbdb200.so`` (CUDA kernels
for sm_100a behind ``include/bdb200.h``); this package holds the deck reader,
the ctypes binding of that library and the build recipe.
"""
__all__ = ["decks"]
