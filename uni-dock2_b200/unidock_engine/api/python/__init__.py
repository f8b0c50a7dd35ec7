from . import pipeline  # noqa: F401
