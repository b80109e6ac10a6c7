"""B200-native SPH particle hot path (neighbour search, WCSPH/PCISPH/IISPH/DFSPH
solver steps) behind the reference's SphBase/WcSph/PciSph/IISph_M/DFSPH
interfaces.  The compute runs in libsphgpu.so (sm_100a CUDA kernels, C ABI in
include/sphgpu.h); this package is the host-side layer over it."""
from .scene import Scene, dam_break, rayleigh_taylor  # noqa: F401
from .sph import (DFSPH, GpuScene, IISph_M, PciSph, SphBase, WcSph, default_params,  # noqa: F401
                  params_for_scene, scene_to_gpu)
