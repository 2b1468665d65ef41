"""vkpathtracer_b200 -- sm_100a render backend for vkPathTracer's CPU hot path.

Public surface:
  CudaPathTracer   the IPathTracer contract over libvkpt_cuda (tracer.py)
  scenes           seeded synthetic scenes and ray sets
  native           ctypes binding of include/vkptc.h
"""
from . import scenes  # noqa: F401
from .scenes import RenderSettings, Scene  # noqa: F401


def __getattr__(name):
    if name in ("CudaPathTracer", "RenderTile", "Status"):
        from . import tracer
        return getattr(tracer, name)
    raise AttributeError(name)
