"""peasoup_b200 -- B200-native acceleration search (Peasoup's per-DM inner
loop) behind Peasoup's transform API.

The compute lives in libpeasoup_b200.so (hand-written sm_100a CUDA + cuFFT)
behind the C ABI of include/peasoup_b200.h.  This package is the Python host
side: ctypes bindings (_lib), the transform-API mirror (transforms), the
search engine and worker loop (search), synthetic inputs (synth) and the
served request loop (served).
"""
from ._lib import PsxError, load  # noqa: F401

__version__ = "0.1.0"


def build(**kw) -> str:
    """Compile the CUDA library in-tree (sm_100a)."""
    from .build import build as _build
    return _build(**kw)
