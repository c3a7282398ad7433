"""astra.projector3d: 'cuda3d' projector objects (python/astra/projector3d.py)."""
from .projector import clear, create, delete, projection_geometry, volume_geometry  # noqa: F401
