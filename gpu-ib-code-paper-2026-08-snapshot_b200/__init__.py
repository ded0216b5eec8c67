"""pyib_b200: B200-native per-step hot path of the PyIB immersed-boundary solver.

The directory name is not a Python identifier, so the package is imported as
``pyib_b200`` through ``_pyib_b200_import.load()`` at the repository root.
"""
__version__ = "0.1.0"
