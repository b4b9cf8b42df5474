"""
pyrecon_b200: pyrecon's reconstruction hot path (MultiGridReconstruction,
IterativeFFTReconstruction, PlaneParallelFFTReconstruction) on NVIDIA B200 GPUs,
through hand-written sm_100a CUDA kernels behind a C ABI (include/pyrecon_cuda.h).
"""
from ._version import __version__
from .mesh import MeshInfo, RealMesh, ComplexMesh, MeshError
from .recon import BaseReconstruction, ReconstructionError
from .multigrid import OriginalMultiGridReconstruction, MultiGridReconstruction
from .iterative_fft import IterativeFFTReconstruction
from .plane_parallel_fft import PlaneParallelFFTReconstruction
from .iterative_fft_particle import OriginalIterativeFFTParticleReconstruction, IterativeFFTParticleReconstruction
from .utils import setup_logging

__all__ = ['MeshInfo', 'RealMesh', 'ComplexMesh', 'MeshError', 'BaseReconstruction', 'ReconstructionError',
           'OriginalMultiGridReconstruction', 'MultiGridReconstruction', 'IterativeFFTReconstruction',
           'PlaneParallelFFTReconstruction', 'OriginalIterativeFFTParticleReconstruction',
           'IterativeFFTParticleReconstruction', 'setup_logging']
