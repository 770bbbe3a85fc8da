"""B200 path tracer: the hot path of pfx's crates/trace as hand-written sm_100a
CUDA kernels behind a C ABI (include/pfxt.h), with a Python mirror of the
reference's `Trace` interface."""
from .trace import (Adaptive, Camera, Converged, Output, Round, SceneBuffers, SceneDesc, Settings, Sun, Trace,
                    TraceError, make_rays)

__all__ = ["Adaptive", "Camera", "Converged", "Output", "Round", "SceneBuffers", "SceneDesc", "Settings", "Sun",
           "Trace", "TraceError", "make_rays"]
