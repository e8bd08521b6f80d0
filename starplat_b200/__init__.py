"""starplat_b200 — B200-native (sm_100a) kernels for StarPlat's static-graph hot path."""
from .graph import CSRGraph  # noqa: F401
