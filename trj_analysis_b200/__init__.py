"""B200-native (sm_100a) species-resolved g_ab(r) and S_ab(Q) for periodic MD frames.

Host code is Python; the arithmetic runs in libtrj_sm100.so (hand-written CUDA for
sm_100a) behind the C ABI of include/trj_sm100.h.  Importing this package does not
touch the GPU; the device layer (``engine``, ``analysis``) loads the library on use
and fails loudly when it is missing.
"""
__version__ = "0.1.0"

from . import frames, refsem  # noqa: F401  (CPU-only modules)
