from . import cache  # noqa: F401
