"""B200-native Flow Lenia step engine.

Hand-written sm_100a CUDA kernels behind a C ABI (include/flowlenia_cuda.h),
with a Python mirror of the reference crate's propagator surface.
"""
from ._native import CONV_AUTO, CONV_DIRECT, CONV_FFT, ConfigError, FlpError
from .adjoint import AdjointBatch, FlowLeniaFunction
from .animation import AnimationPlayer, AnimationRecorder
from .batch import BatchedPropagator
from .embedded import EmbeddedPropagator, EmbeddedState
from .propagator import CudaPropagator, SimulationConfig, SimulationState

__all__ = ["AdjointBatch", "AnimationPlayer", "AnimationRecorder", "FlowLeniaFunction", "BatchedPropagator", "EmbeddedPropagator", "EmbeddedState", "CudaPropagator", "SimulationConfig", "SimulationState", "ConfigError", "FlpError", "CONV_AUTO",
           "CONV_DIRECT", "CONV_FFT"]
