"""bem-mececcs_b200: B200-native BEM hot path (H/G assembly + complex LU solve)."""
from . import formats, meshgen  # noqa: F401
