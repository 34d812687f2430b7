"""B200 implementation of GeoBrain's 2-D acoustic wave path.

Drop-in for the acoustic part of ``geobrain.physics.wave``:

    from geobrain_b200 import wave
    grid = wave.GridConfig(nx=200, nz=100, dx=10, dz=10)
    model = wave.AcousticModel(grid, wave.BoundaryConfig(n_layers=20), vp=vp, rho=rho, vp_grad=True,
                               device="cuda")
    prop = wave.AcousticPropagator(model, survey, device="cuda")
    result = prop.forward(checkpoint_segments=4)     # result.p: (n_shots, nt, n_receivers)

Same class and function names, arguments and results as the reference for
GridConfig, BoundaryConfig, TimeConfig, WaveletConfig, SolverConfig,
AbstractModel, AcousticModel, AbstractPropagator, AcousticPropagator,
WaveResult, Source, Receiver, Survey, RickerWavelet, GaussianWavelet,
create_wavelet, bc_pml, create_boundary and kernels.acoustic_forward_kernel /
kernels.pad_model; the compute runs in hand-written sm_100a CUDA kernels.
"""
from . import kernel as kernels
from . import misfit, sharding
from .batched import AcousticBatch, acoustic_forward_batched, acoustic_gradient_batched
from .boundary import bc_pml, bc_pml_3d, create_boundary
from .config import BoundaryConfig, GridConfig, SolverConfig, TimeConfig, WaveletConfig
from .kernel import acoustic_forward_kernel, pad_model
from .kernel3d import acoustic_forward_kernel_3d, pad_model_3d
from .model import UNITS, AbstractModel, AcousticModel, numpy2tensor
from .propagator import AbstractPropagator, AcousticPropagator
from .result import WaveResult
from .survey import Receiver, Source, Survey
from .wavelet import GaussianWavelet, RickerWavelet, WaveletGenerator, create_wavelet

__all__ = [
    "GridConfig", "BoundaryConfig", "TimeConfig", "WaveletConfig", "SolverConfig",
    "AbstractModel", "AbstractPropagator", "WaveResult", "UNITS", "AcousticModel",
    "WaveletGenerator", "RickerWavelet", "GaussianWavelet", "create_wavelet",
    "bc_pml", "create_boundary", "Source", "Receiver", "Survey", "AcousticPropagator",
    "numpy2tensor", "kernels", "acoustic_forward_kernel", "pad_model",
    "AcousticBatch", "acoustic_forward_batched", "acoustic_gradient_batched", "sharding", "misfit",
    "acoustic_forward_kernel_3d", "pad_model_3d", "bc_pml_3d",
]
