"""grasph_b200 — host-side mirror of Grasph.jl's SPH API over libgrasph_cuda.so.

The per-timestep hot path (cell-key sort, CSR grid, ghosts, staged pair
sweeps, state updaters, leapfrog update) runs as sm_100a CUDA kernels behind
the C ABI in include/grasph_cuda.h; this package builds the model through
that ABI and moves host arrays in and out.
"""
from . import consts
from .model import (AbstractParticleSystem, ArgumentError, BasicParticleSystem, CauchyFluidPfn,
                    CountingPfn, CubicSplineKernel, DynamicBoundarySystem, ElastoPlasticParticleSystem,
                    ElastoPlasticStressUpdater, FluidParticleSystem, FluidPfn, FluidSolidPfn, GhostCopier, GhostEntry,
                    GhostParticleSystem, HookeLawStressUpdater, HouseholderReflect, LeapFrogTimeIntegrator, RK4TimeIntegrator,
                    LinearEOSUpdater, StaticBoundarySystem, StrainRatePfn, StrainRateVorticityPfn,
                    StressParticleSystem, SystemInteraction, TaitEOSUpdater, ViscoPlasticMCStressUpdater,
                    WenlandC2Kernel, XSPHPfn, ZeroFieldUpdater, is_coupled, VirtualParticleSystem,
                    InterpolateFieldFn, VirtualNormUpdater, PrescribedVelocityUpdater, ProbeParticleSystem,
                    NeighborCountFn, float_type)
from .engine import (CudaBackend, GcError, Server, Session, compile_instance, download_instance, load_library,
                     time_integrate, upload_instance)

PRECISION_FP64 = consts.GC_PRECISION_FP64
PRECISION_FP32_COMPENSATED = consts.GC_PRECISION_FP32_COMPENSATED
