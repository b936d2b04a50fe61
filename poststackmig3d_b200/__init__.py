"""poststackmig3d_b200: B200-native Kirchhoff post-stack 3D time migration.

The diffraction summation of sergeevsn/poststackmig3d (src/migration_kernel.cpp) rebuilt as
hand-written sm_100a CUDA behind a C ABI (include/psm.h), with the reference's host surface
(config.txt keys, SEG-Y IBM/IEEE I/O with INLINE_3D/CROSSLINE_3D lookup, padding, Vrms from
SEG-Y / table / constant) in C++ (include/psm_host.h).
"""
from .migration import (Batch, Geometry, MigrationKernel, Migrator, Problem,  # noqa
                        estimate_max_velocity,
                        max_aperture_il, output_centers, padded_labels, plan_geometry,
                        tan2_theta)

__all__ = ["Batch", "Geometry", "MigrationKernel", "Migrator", "Problem",
           "estimate_max_velocity",
           "max_aperture_il", "output_centers", "padded_labels", "plan_geometry",
           "tan2_theta"]
