"""B200-native (sm_100a) SOAP/GAP energy-and-force path: a drop-in for TurboGAP's
predict / md / mc hot path (neighbor list, soap_turbo descriptor, GAP prediction).

The compute path is libtgap.so (hand-written CUDA for sm_100a behind the C ABI of
include/tgap.h); this package is the host-side mirror of the reference interface.
"""
import importlib

from . import gap_file, screen, synth, xyz  # noqa: F401
from .native import TGAP_FP64, TGAP_MIXED, TgapError, LIB_PATH  # noqa: F401


def __getattr__(name):
    # the GPU API loads libtgap.so on first use and raises if it is missing
    if name in ("Context", "Model", "System", "MD", "MC", "Terms", "assign_species", "api"):
        api = importlib.import_module(__name__ + ".api")
        return api if name == "api" else getattr(api, name)
    raise AttributeError(name)
