"""B200-native escape-time engine: drop-in for the render entry points of
math_core/engine.py (Apeiron).  See fractura_b200.engine."""
from .config import RenderParameters  # noqa: F401

__all__ = ["RenderParameters", "engine"]
