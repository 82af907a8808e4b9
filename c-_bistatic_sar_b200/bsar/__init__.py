"""bsar -- B200 bistatic SAR back-projection (host side of libbsar.so).

``bsar.native``  ctypes binding of the C ABI in include/bsar.h (the product path)
``bsar.scene``   seeded synthetic scenes of the benchmark configurations
"""
from . import native, scene  # noqa: F401
from .native import BsarError, Context, DemArrays, Server, submit_scene, synthesize_scene, upload_scene  # noqa: F401

__all__ = ["native", "scene", "Context", "DemArrays", "BsarError", "Server", "submit_scene", "upload_scene",
           "synthesize_scene"]
