"""Boundary-condition and interpolation-order enums.

Same member names, aliases and integer values as the enums that
nitorch's compiled backend exports (nitorch/_C/spatial.cpp:48-73, values
from nitorch/_C/src/bounds.h and interpolation.h).  Like the pybind11 enums
they are not integers: ``BoundType.zero == 7`` is False, ``int(b)`` and
``b.value`` give the code.
"""
import enum


class _CodeEnum(enum.Enum):
    def __int__(self):
        return self.value

    def __index__(self):
        return self.value

    def __repr__(self):
        return f"<{type(self).__name__}.{self.name}: {self.value}>"


class BoundType(_CodeEnum):
    """Boundary conditions (pad modes) of the spline sampling path."""
    replicate = 0     #  a  a  a | a b c d |  d  d  d
    nearest = 0
    dct1 = 1          #  d  c  b | a b c d |  c  b  a
    mirror = 1
    dct2 = 2          #  c  b  a | a b c d |  d  c  b
    reflect = 2
    dst1 = 3          # -b -a  0 | a b c d |  0 -d -c
    antimirror = 3
    dst2 = 4          # -c -b -a | a b c d | -d -c -b
    antireflect = 4
    dft = 5           #  b  c  d | a b c d |  a  b  c
    wrap = 5
    zero = 7          #  0  0  0 | a b c d |  0  0  0


class InterpolationType(_CodeEnum):
    """B-spline interpolation orders."""
    nearest = 0
    linear = 1
    quadratic = 2
    cubic = 3
    fourth = 4
    fifth = 5
    sixth = 6
    seventh = 7


class GridAlignType(_CodeEnum):
    """Lattice alignment of nitorch's native resize (nitorch/_C/src/
    grid_align.h:7-12; values as the compiled backend exports them)."""
    edge = 0      # outer edges of the corner voxels
    center = 1    # centres of the corner voxels
    first = 2     # centre of the first voxel (factor kept)
    last = 3      # centre of the last voxel (factor kept)


# Prefilter integer bound codes (nitorch/_C/_ts/bounds.py:7-14), used by the
# interpol-compatible spline_coeff entry points.
TS_BOUND = {BoundType.zero: 0, BoundType.replicate: 1, BoundType.dct1: 2,
            BoundType.dct2: 3, BoundType.dst1: 4, BoundType.dst2: 5,
            BoundType.dft: 6}
