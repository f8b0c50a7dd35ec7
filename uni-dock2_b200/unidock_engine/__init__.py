"""Drop-in package path of the reference engine's Python module (unidock_engine.api.python)."""
