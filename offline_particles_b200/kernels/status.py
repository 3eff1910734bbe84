"""Particle status codes (kernels/status.pxd:1-14, status.pyx:8-21 of the reference)."""

from enum import IntEnum

INACTIVE = 0x80
NORMAL = 0
NONFINITE = 1 | INACTIVE
OUT_OF_DOMAIN = 2 | INACTIVE
MULTISTEP_1 = 10
MULTISTEP_2 = 11


class ParticleStatus(IntEnum):
    # inactive flag (bit 7): every kernel skips particles that carry it
    INACTIVE = INACTIVE
    # normal state
    NORMAL = NORMAL
    # error states
    NONFINITE = NONFINITE
    OUT_OF_DOMAIN = OUT_OF_DOMAIN
    # reserved for multistep initialisation (AB3 bootstrap)
    MULTISTEP_1 = MULTISTEP_1
    MULTISTEP_2 = MULTISTEP_2
