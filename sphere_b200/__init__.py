"""sphere_b200: a B200-native (sm_100a) DEM time step behind the drop-in
surface of 19revey/sphere's python/sphere.py (the ``sim`` class, the .bin
v2.15 format and ``run()``)."""
from .sim import VERSION, V_sphere, cleanup, convert, render, sim, status  # noqa: F401

__all__ = ["sim", "status", "cleanup", "render", "convert", "V_sphere", "VERSION"]
