"""bsnn -- Python interface of libbsnn, the B200-native engine for the per-step hot path of the
paulazoo/example-cuda-spiking-nn simulator (System::step_the_clock).

The compute path is the CUDA library libbsnn.so; this package only wraps its C-ABI
(include/bsnn.h) with ctypes and builds networks.  Importing it does not load the library;
creating a Simulation does, and fails loudly if libbsnn.so is missing.
"""
from ._ffi import (FIELD, NOISE_OFF, NOISE_PHILOX, NOISE_REPLAY, PLASTICITY_ISTDP, PLASTICITY_STDP, PLASTICITY_TRIPLET,
                   WEIGHT_FORMATS,
                   BsnnError, ConnectionParams, ConnectionView, CudaError, DeviceTimeout, InvalidArgument, NeuronGroupParams,
                   OutOfRange, PlasticityParams, StateError, load_library)
from .adjoint import AdjointNetwork, config5_network, spiking_loss_function
from .batch import BatchSimulation, BatchSpec, config4_batch
from .core import Simulation, connection_propagate
from .network import NetworkSpec, random_network, synthetic_network

__all__ = [
    "FIELD", "WEIGHT_FORMATS", "NOISE_OFF", "NOISE_PHILOX", "NOISE_REPLAY", "PLASTICITY_ISTDP", "PLASTICITY_STDP", "PLASTICITY_TRIPLET",
    "BsnnError", "ConnectionParams", "ConnectionView", "CudaError", "DeviceTimeout", "InvalidArgument", "NeuronGroupParams",
    "OutOfRange", "PlasticityParams", "StateError", "load_library", "Simulation", "BatchSimulation", "BatchSpec",
    "config4_batch", "AdjointNetwork", "config5_network", "spiking_loss_function", "connection_propagate", "NetworkSpec", "random_network",
    "synthetic_network",
]
