"""Fieldset: the named fields and constants of a simulation (fieldset.py:11-241 of the reference)."""

from __future__ import annotations

import types
from typing import Any, ItemsView, KeysView, Mapping, ValuesView

import numpy as np

from .fields import Field


class Fieldset:
    """A collection of fields on a ``(t, z, y, x)`` grid of centred sizes, plus constants.

    Index bounds default to ``(0, N - 1)`` per dimension and are registered as
    the constants ``zidx_min`` ... ``xidx_max`` that the validation kernel reads.
    """

    def __init__(
        self,
        t_size: int,
        z_size: int,
        y_size: int,
        x_size: int,
        *,
        constants: Mapping[str, Any] | None = None,
        zidx_bounds: tuple[float, float] | None = None,
        yidx_bounds: tuple[float, float] | None = None,
        xidx_bounds: tuple[float, float] | None = None,
        **fields: Field,
    ) -> None:
        self._t_size = t_size
        self._z_size = z_size
        self._y_size = y_size
        self._x_size = x_size
        if zidx_bounds is None:
            zidx_bounds = (0, z_size - 1)
        if yidx_bounds is None:
            yidx_bounds = (0, y_size - 1)
        if xidx_bounds is None:
            xidx_bounds = (0, x_size - 1)
        self._zidx_bounds = (np.float64(zidx_bounds[0]), np.float64(zidx_bounds[1]))
        self._yidx_bounds = (np.float64(yidx_bounds[0]), np.float64(yidx_bounds[1]))
        self._xidx_bounds = (np.float64(xidx_bounds[0]), np.float64(xidx_bounds[1]))
        self._fields: dict[str, Field] = {}
        self._constants: dict[str, Any] = {}
        if constants is not None:
            for name, value in constants.items():
                self.add_constant(name, value)
        self.add_constant("zidx_min", self._zidx_bounds[0])
        self.add_constant("zidx_max", self._zidx_bounds[1])
        self.add_constant("yidx_min", self._yidx_bounds[0])
        self.add_constant("yidx_max", self._yidx_bounds[1])
        self.add_constant("xidx_min", self._xidx_bounds[0])
        self.add_constant("xidx_max", self._xidx_bounds[1])
        for name, field in fields.items():
            self.add_field(name, field)

    @property
    def t_size(self) -> int:
        return self._t_size

    @property
    def z_size(self) -> int:
        return self._z_size

    @property
    def y_size(self) -> int:
        return self._y_size

    @property
    def x_size(self) -> int:
        return self._x_size

    @property
    def zidx_bounds(self) -> tuple[float, float]:
        return self._zidx_bounds

    @property
    def yidx_bounds(self) -> tuple[float, float]:
        return self._yidx_bounds

    @property
    def xidx_bounds(self) -> tuple[float, float]:
        return self._xidx_bounds

    @property
    def zidx_min(self) -> float:
        return self._zidx_bounds[0]

    @property
    def zidx_max(self) -> float:
        return self._zidx_bounds[1]

    @property
    def yidx_min(self) -> float:
        return self._yidx_bounds[0]

    @property
    def yidx_max(self) -> float:
        return self._yidx_bounds[1]

    @property
    def xidx_min(self) -> float:
        return self._xidx_bounds[0]

    @property
    def xidx_max(self) -> float:
        return self._xidx_bounds[1]

    @property
    def simulation_shape(self) -> tuple[int, int, int, int]:
        return (self._t_size, self._z_size, self._y_size, self._x_size)

    @property
    def fields(self) -> Mapping[str, Field]:
        return types.MappingProxyType(self._fields)

    @property
    def constants(self) -> Mapping[str, Any]:
        return types.MappingProxyType(self._constants)

    def add_field(self, name: str, field: Field) -> None:
        if name in self:
            raise KeyError(f"Field '{name}' already exists in Fieldset. First remove it before adding a new one.")
        try:
            field.validate_shape(self.simulation_shape)
        except ValueError as e:
            raise ValueError(f"Error validating shape of Field '{name}'.") from e
        self._fields[name] = field

    def add_constant(self, name: str, value: Any) -> None:
        if name in self._constants or name in self:
            raise KeyError(f"'{name}' already exists in Fieldset. First remove it before adding a new one.")
        self._constants[name] = _numpyify_constant(value)

    def remove(self, name: str) -> None:
        if name in self._constants:
            del self._constants[name]
            return
        if name in self._fields:
            del self._fields[name]
            return
        raise KeyError(f"Field '{name}' does not exist in Fieldset. Cannot remove.")

    def __getitem__(self, name: str) -> Field:
        if name in self._fields:
            return self._fields[name]
        raise KeyError(f"Field '{name}' does not exist in Fieldset.")

    def __contains__(self, name: str) -> bool:
        return name in self._fields

    def keys(self) -> KeysView[str]:
        return self._fields.keys()

    def values(self) -> ValuesView[Field]:
        return self._fields.values()

    def items(self) -> ItemsView[str, Field]:
        return self._fields.items()

    def __repr__(self) -> str:
        field_str = ", \n\t".join(f"{key} = {value}" for key, value in self._fields.items())
        return (f"Fieldset(\n\tt_size={self.t_size}, z_size={self.z_size}, y_size={self.y_size}, "
                f"x_size={self.x_size},\n\tconstants={self._constants}, \n\t{field_str}\n)")


def _numpyify_constant(value: Any):
    """A single value as a Python scalar (fieldset.py:233-241)."""
    try:
        arr = np.asarray(value)
        if arr.size != 1:
            raise ValueError(f"Expected a single value, got array of size {arr.size}.")
        return arr.item()
    except (ValueError, TypeError) as e:
        raise ValueError(f"Cannot convert value '{value}' to a numpy scalar.") from e
