"""Host-side mirror of tigre.utilities for the projector-pair path."""
from .geometry import Geometry, ParallelGeo, geometry, ConeGeometryDefault, cone_geometry  # noqa: F401
