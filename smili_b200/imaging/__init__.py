"""Imaging drivers (static)."""
from . import lbfgs  # noqa: F401
