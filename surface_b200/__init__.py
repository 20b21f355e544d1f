"""surface_b200 -- B200-native LBVH build, closest-hit traversal and volume
march with the interface of SURFACE's render/ accel classes.

The compute path is libsurface_rt.so (hand-written sm_100a CUDA behind the C
ABI of include/surface_rt.h); this package is its host-side mirror.
"""
from .accel import (HIT_DTYPE, MISS, RAY_DTYPE, Context, Mesh, ParticleAccel,  # noqa: F401
                    ParticleBuildOptions, Particles, SurfaceError, Tetrahedron,
                    TetraAccel, TetraBuildOptions, TriangleAccel, TriangleBuildOptions,
                    spawn_secondary, stage_karras, stage_morton, stage_sort_pairs)
from .lines import LineAccel, LineBuildOptions, Lines  # noqa: F401
from .solids import Solid, SolidAccel  # noqa: F401
