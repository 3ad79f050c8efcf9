"""uv-table helpers used by the imaging drivers."""
from . import tools  # noqa: F401
