"""simulatokit_b200: SimulatoKit's multislice hot path as a B200-native CUDA library (libsimulato_cuda.so) with a
host-side mirror of SimulatoKit's API (Multislice.run / runBatch, STEM.scan, Potential, Probe, detectors).

The CUDA library is the product; these modules validate arguments, prepare the host-side inputs the reference's
Swift types prepare, and call the C ABI. There is no CPU fallback: without the built library or an sm_100 device
every compute call raises CudaUnavailable."""

from ._lib import CudaFailure, CudaUnavailable, InvalidArgument, SimulatoError  # noqa: F401
from .core import Antialias, AtomicStructure, ElectronBeam, Grid, Waves  # noqa: F401
from .detector import (STEM, AnnularDetector, BinnedPixelatedDetector, CenterOfMassDetector,  # noqa: F401
                       PixelatedDetector, RealField, ScanMeasurement, ScanWaves, SegmentedDetector, WavesDetector,
                       detector_shape)
from .engine import Engine, ExecutionOptions  # noqa: F401
from .multislice import (Backend, ExitPlanes, FrozenPhonons, GaussianGenerator, JobTable,  # noqa: F401
                         LobatoParameterization, Multislice, Potential, ProjectedPotential, Slicing, Surrogate,
                         TiledPotential, finite_profile)
from .probe import Aberrations, Aperture, ContrastTransferFunction, GridScan, Probe  # noqa: F401
