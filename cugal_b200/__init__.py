"""B200-native FUGAL graph alignment: a drop-in for cuGAL's ``cugal()`` + ``Config``.

Use ``cugal`` to run the algorithm (reference ``cugal/__init__.py:1-7``).
"""

from .config import Config, HungarianMethod, SinkhornMethod  # noqa: F401
from .pred import cugal  # noqa: F401
from .profile import Phase, Profile, SinkhornProfile, TimeStamp  # noqa: F401
