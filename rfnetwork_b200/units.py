"""Physical constants and unit conversions used by the FDTD setup.

Same values as the reference (rfnetwork/core/units.py:3-124): geometry is in
inches and converted to metres with ``conv.m_in`` (a multiply by 1/39.3701).
"""
import numpy as np


class const:
    c0 = 299792458
    e0 = 8.854187817e-12
    u0 = 4 * np.pi * 1e-7
    eta0 = np.sqrt(u0 / e0)


class conv:
    """``<to>_<from>`` ratio conversions; only the ones the FDTD path needs."""

    _in_m = 39.3701

    @staticmethod
    def in_m(v):
        return 39.3701 * v

    @staticmethod
    def m_in(v):
        return (1 / 39.3701) * v

    @staticmethod
    def mm_in(v):
        return 25.4 * v

    @staticmethod
    def in_mm(v):
        return (1 / 25.4) * v
