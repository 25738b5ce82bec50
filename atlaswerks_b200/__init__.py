"""atlaswerks_b200 — B200-native (sm_100a) greedy-fluid / LDMM registration
inner loop behind the AtlasWerks iterator and kernel interfaces.

The compute path is libaw_b200.so (C ABI: include/aw_b200.h); this package
is the host-side mirror of the reference interfaces over that ABI, plus the
seeded synthetic workload generators.
"""
from ._lib import AwError, build  # noqa: F401

__version__ = "0.1.0"
