"""Seeded synthetic media and sources of the benchmark configurations.

The generators belong to the library (helm3d.media: they make the inputs of
its benchmark and examples); the oracle checks solves of the same Problem
objects, so it re-exports them here for the tests.
"""
from helm3d.media import *  # noqa: F401,F403
from helm3d.media import Problem, SplitMix64, anomalies, gaussian_source, layered_medium  # noqa: F401
