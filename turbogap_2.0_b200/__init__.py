"""B200-native SOAP/GAP energy-and-force path (TurboGAP drop-in), host-side package."""
from . import synth  # noqa: F401
