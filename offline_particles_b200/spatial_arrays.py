"""Grid staggering and device-resident spatial arrays.

``Stagger`` keeps the reference's names and semantics (spatial_arrays.py:18-68
of offline_particles): a field's index along a dimension is the centred
(rho-point) index plus ``offset``, and its size follows ``expected_size``.

``DeviceArray`` plays the part of the reference's ``NumpyArray``
(spatial_arrays.py:182-225): the whole array is resident -- here in HBM -- and
``get_data_subset`` ignores the bounding box, returning the array with its
active offsets.  The reference's dask path (``ChunkedDaskArray``,
spatial_arrays.py:228-351) loads a padded bounding-box subset per launch; on a
180 GB device the fields stay whole, so it has no counterpart here.
"""

from __future__ import annotations

import collections
import enum

import numpy as np

BBox = collections.namedtuple("BBox", ("zmin", "zmax", "ymin", "ymax", "xmin", "xmax"))


@enum.unique
class Stagger(enum.StrEnum):
    """Staggering of one grid dimension (Arakawa-C)."""

    CENTER = "center"
    LEFT = "left"
    RIGHT = "right"
    INNER = "inner"
    OUTER = "outer"
    INVARIANT = "invariant"

    @property
    def offset(self) -> float | None:
        """Offset added to a centred index to get this stagger's index."""
        if self is Stagger.CENTER:
            return 0.0
        if self in (Stagger.LEFT, Stagger.OUTER):
            return 0.5
        if self in (Stagger.RIGHT, Stagger.INNER):
            return -0.5
        return None

    def expected_size(self, N: int) -> int | None:
        """Size of this dimension given the centred size ``N``."""
        if self in (Stagger.CENTER, Stagger.LEFT, Stagger.RIGHT):
            return N
        if self is Stagger.OUTER:
            return N + 1
        if self is Stagger.INNER:
            return N - 1
        return None

    @property
    def is_invariant(self) -> bool:
        return self is Stagger.INVARIANT

    @property
    def is_active(self) -> bool:
        return self is not Stagger.INVARIANT

    @property
    def on_face(self) -> bool:
        return self in {Stagger.LEFT, Stagger.RIGHT, Stagger.INNER, Stagger.OUTER}

    @property
    def at_center(self) -> bool:
        return self is Stagger.CENTER


class SpatialArray:
    """Base: an array over the active dimensions of a (z, y, x) stagger."""

    def __init__(self, z_stagger: Stagger, y_stagger: Stagger, x_stagger: Stagger) -> None:
        self._z_stagger = Stagger(z_stagger)
        self._y_stagger = Stagger(y_stagger)
        self._x_stagger = Stagger(x_stagger)

    @property
    def z_stagger(self) -> Stagger:
        return self._z_stagger

    @property
    def y_stagger(self) -> Stagger:
        return self._y_stagger

    @property
    def x_stagger(self) -> Stagger:
        return self._x_stagger

    @property
    def stagger(self) -> tuple[Stagger, Stagger, Stagger]:
        return (self._z_stagger, self._y_stagger, self._x_stagger)

    @property
    def offsets(self) -> tuple[float | None, float | None, float | None]:
        return tuple(s.offset for s in self.stagger)  # type: ignore[return-value]

    @property
    def dmask(self) -> tuple[bool, bool, bool]:
        return tuple(s.is_active for s in self.stagger)  # type: ignore[return-value]

    @property
    def active_offsets(self) -> tuple[float, ...]:
        return tuple(s.offset for s in self.stagger if s.is_active)  # type: ignore[misc]


class DeviceArray(SpatialArray):
    """A spatial array held whole on the device (a ``torch.Tensor`` on CUDA)."""

    def __init__(self, data, z_stagger: Stagger, y_stagger: Stagger, x_stagger: Stagger, *, dtype=None,
                 device=None) -> None:
        super().__init__(z_stagger, y_stagger, x_stagger)
        import torch

        from ._device import cuda_device

        dev = cuda_device(device)
        t = data if isinstance(data, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(np.asarray(data)))
        if dtype is not None:
            t = t.to(dtype)
        self._data = t.to(dev).contiguous()

    @property
    def data(self):
        return self._data

    @property
    def dtype(self) -> np.dtype:
        from ._device import numpy_dtype

        return numpy_dtype(self._data.dtype)

    @property
    def shape(self) -> tuple[int, ...]:
        return tuple(self._data.shape)

    def get_data_subset(self, bounding_box: BBox | None = None):
        """The whole array and its active offsets (the bounding box is not needed)."""
        return self._data, self.active_offsets


class NumpyArray(DeviceArray):
    """Constructor-compatible stand-in for the reference's ``NumpyArray``: the
    host array is copied to the device once and kept whole."""

    def __init__(self, data, z_stagger: Stagger, y_stagger: Stagger, x_stagger: Stagger) -> None:
        super().__init__(np.asarray(data), z_stagger, y_stagger, x_stagger)
