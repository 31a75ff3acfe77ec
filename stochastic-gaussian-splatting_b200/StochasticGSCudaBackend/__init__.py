"""B200-native drop-in for the reference's StochasticGSCudaBackend (per-sample stochastic render path)."""
from .render import render, Settings, TemporalMode, History, create_k_buffer
__all__ = ['render', 'Settings', 'TemporalMode', 'History', 'create_k_buffer']
