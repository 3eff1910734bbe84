"""Simulation output (output/_output.py, output/_linear_interpolation.py of the reference).

``Output``, ``AbstractOutputWriter``, ``AbstractOutputWriterBuilder`` and
``linearly_interpolate_fields`` keep the reference's API: a writer turns its
outputs into events (time, each output, a round check) that the simulation
fires on its schedule.

The reference's writer stores rows in a zarr store (output/_zarr_writer.py),
and zarr is not part of this package's environment.  ``NpyOutputBuilder``
writes the same rows — a time array ``(rounds,)`` and one ``(rounds,
nparticles)`` array per output, particles in their original order — as
``.npy`` files in a directory.  A row leaves the device with an asynchronous
copy into pinned host memory, and a background thread appends it to its file
once the copy is done, so writing overlaps the next launches instead of
stopping the device at every output event.
"""

from __future__ import annotations

import abc
import concurrent.futures
import functools
import os
import types
from pathlib import Path
from typing import Mapping

import numpy as np
import torch

from ..events import Event, SimulationState
from ..fieldset import Fieldset
from ..kernels import ParticleKernel, merge_particle_fields
from ..kernels.output import bilinear_interpolation_kernel, linear_interpolation_kernel, trilinear_interpolation_kernel


class Output:
    """One output: a particle field filled by ``kernels`` (output/_output.py:14-41)."""

    __slots__ = ("name", "particle_field", "dtype", "kernels")

    def __init__(self, name: str, *kernels: ParticleKernel, particle_field: str | None = None) -> None:
        if particle_field is None:
            particle_field = name
        fields = merge_particle_fields(kernels)
        if particle_field not in fields:
            raise ValueError(f"Particle field '{particle_field}' not found in provided kernels.")
        object.__setattr__(self, "name", name)
        object.__setattr__(self, "particle_field", particle_field)
        object.__setattr__(self, "dtype", np.dtype(fields[particle_field]))
        object.__setattr__(self, "kernels", tuple(kernels))

    def __setattr__(self, name, value):
        raise AttributeError("Output is immutable")

    def __repr__(self) -> str:
        return f"Output(name={self.name!r}, particle_field={self.particle_field!r}, dtype={self.dtype})"


class AbstractOutputWriter(abc.ABC):
    """Interface of output writers (output/_output.py:44-117)."""

    @property
    @abc.abstractmethod
    def name(self) -> str: ...

    @property
    @abc.abstractmethod
    def outputs(self) -> Mapping[str, Output]: ...

    @abc.abstractmethod
    def write_time(self, state: SimulationState) -> None: ...

    @abc.abstractmethod
    def write_output(self, name: str, state: SimulationState) -> None: ...

    @abc.abstractmethod
    def finalise_write_round(self, state: SimulationState) -> None: ...

    def event_name(self, output_name: str) -> str:
        return f"{self.name}:{output_name}"

    def create_events(self) -> list[Event]:
        """Events in firing order: the time, each output (after its kernels), the round check.  The events
        are deferrable (they may fire after a fused launch on the state recorded at their step) when every
        output's kernels only sample fields into fields of their own."""
        from .. import _lib
        from ..kernels.output.linear_interpolation import samples_only

        step_fields = {"status", "rho_t", *_lib.PARTICLE_POINTERS}
        defer = all(samples_only(k, step_fields) for o in self.outputs.values() for k in o.kernels)
        events = [Event(self.event_name("time"), self.write_time, deferrable=defer)]
        for name, output in self.outputs.items():
            events.append(Event(self.event_name(name), functools.partial(self.write_output, name), *output.kernels,
                                deferrable=defer))
        events.append(Event(self.event_name("finalise"), self.finalise_write_round, deferrable=defer))
        return events


class AbstractOutputWriterBuilder(abc.ABC):
    """Interface of output-writer builders (output/_output.py:120-158)."""

    @property
    @abc.abstractmethod
    def name(self) -> str: ...

    @property
    @abc.abstractmethod
    def outputs(self) -> Mapping[str, Output]: ...

    @abc.abstractmethod
    def add_output(self, *outputs: Output, **kwargs) -> None: ...

    @abc.abstractmethod
    def remove_output(self, name: str) -> None: ...

    @abc.abstractmethod
    def build(self, nparticles: int, time_type: np.dtype) -> AbstractOutputWriter: ...


_DMASK_DIMS_2D = {(True, True, False): ("z", "y"), (True, False, True): ("z", "x"), (False, True, True): ("y", "x")}


def linearly_interpolate_fields(fieldset: Fieldset, *variables: str,
                                particle_field_prefix: str = "_output") -> list[Output]:
    """Outputs that sample fields at the particles by linear interpolation
    (output/_linear_interpolation.py:18-56): one kernel per variable, writing a particle field shared by
    the variables of one dtype (each output event runs its kernel just before writing)."""
    dims = ("z", "y", "x")
    outputs = []
    for var in variables:
        if var not in fieldset:
            raise KeyError(f"Field '{var}' not found in fieldset.")
        field = fieldset[var]
        dmask = field.dmask
        ndim = field.nspatial_dims
        particle_field = f"{particle_field_prefix}_{field.dtype}"
        if ndim == 1:
            kernel = linear_interpolation_kernel(var, particle_field, dims[dmask.index(True)])
        elif ndim == 2:
            kernel = bilinear_interpolation_kernel(var, particle_field, _DMASK_DIMS_2D[dmask])
        elif ndim == 3:
            kernel = trilinear_interpolation_kernel(var, particle_field)
        else:
            raise ValueError(f"Field '{var}' has unsupported number of dimensions: {ndim}")
        outputs.append(Output(var, kernel, particle_field=particle_field))
    return outputs


class _RowFile:
    """Rows of one array appended to a raw file; ``.npy`` with a header when the writer closes."""

    def __init__(self, path: Path, row_shape: tuple[int, ...], dtype: np.dtype) -> None:
        self.path = path
        self.raw = path.with_suffix(".raw")
        self.row_shape = row_shape
        self.dtype = np.dtype(dtype)
        self.rows = 0
        self.fh = open(self.raw, "wb")

    def append(self, row: np.ndarray) -> None:
        self.fh.write(np.ascontiguousarray(row, dtype=self.dtype).tobytes())
        self.rows += 1

    def read(self) -> np.ndarray:
        self.fh.flush()
        return np.fromfile(self.raw, dtype=self.dtype).reshape((self.rows,) + self.row_shape)

    def close(self) -> None:
        self.fh.close()
        out = np.lib.format.open_memmap(self.path, mode="w+", dtype=self.dtype, shape=(self.rows,) + self.row_shape)
        if self.rows:
            out[...] = np.fromfile(self.raw, dtype=self.dtype).reshape(out.shape)
        out.flush()
        del out
        os.remove(self.raw)


class NpyOutputWriter(AbstractOutputWriter):
    """Rows of the time and every output, appended as the simulation fires its output events."""

    def __init__(self, name: str, directory: Path, time_name: str, time_type: np.dtype,
                 outputs: Mapping[str, Output], nparticles: int) -> None:
        self._name = name
        self._dir = directory
        self._outputs = types.MappingProxyType(dict(outputs))
        self._time = _RowFile(directory / f"{time_name}.npy", (), time_type)
        self._files = {n: _RowFile(directory / f"{n}.npy", (nparticles,), o.dtype) for n, o in outputs.items()}
        self._count = 0  # completed rounds
        self._written: dict[str, int] = {n: 0 for n in outputs}
        self._times = 0
        self._pool = concurrent.futures.ThreadPoolExecutor(max_workers=1, thread_name_prefix="opb-output")
        self._pending: list[concurrent.futures.Future] = []
        self._closed = False

    @property
    def name(self) -> str:
        return self._name

    @property
    def directory(self) -> Path:
        return self._dir

    @property
    def outputs(self) -> Mapping[str, Output]:
        return self._outputs

    def write_time(self, state: SimulationState) -> None:
        t = np.array([state.time]).astype(self._time.dtype)[0]
        self._pending.append(self._pool.submit(self._time.append, t))
        self._times += 1

    def write_output(self, name: str, state: SimulationState) -> None:
        if name not in self._outputs:
            raise KeyError(f"Output variable '{name}' not found.")
        field = self._outputs[name].particle_field
        dev = state.particles.device_original(field)  # original particle order, on the device
        host = torch.empty(dev.shape, dtype=dev.dtype, pin_memory=True)
        host.copy_(dev, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(dev.device))
        f = self._files[name]

        def land(host=host, ev=ev, f=f) -> None:
            ev.synchronize()
            f.append(host.numpy())

        self._pending.append(self._pool.submit(land))
        self._written[name] += 1

    def finalise_write_round(self, state: SimulationState) -> None:
        """Every output has one more row than at the last round (output/_zarr_writer.py:74-90)."""
        expected = self._count + 1
        if self._times != expected:
            raise RuntimeError(f"Time output has {self._times} entries, expected {expected}.")
        for name, n in self._written.items():
            if n != expected:
                raise RuntimeError(f"Output '{name}' has {n} time entries, expected {expected}.")
        self._count += 1
        self._pending = [f for f in self._pending if not f.done()]

    def flush(self) -> None:
        """Wait until every row written so far is in its file."""
        for f in self._pending:
            f.result()
        self._pending = []

    def read(self, name: str) -> np.ndarray:
        """The rows of output ``name`` (or of the time array, under its name) written so far."""
        self.flush()
        if name == self._time.path.stem:
            return self._time.read()
        return self._files[name].read()

    def close(self) -> None:
        """Flush and turn the row files into ``.npy`` files."""
        if self._closed:
            return
        self.flush()
        self._pool.shutdown(wait=True)
        self._time.close()
        for f in self._files.values():
            f.close()
        self._closed = True


class NpyOutputBuilder(AbstractOutputWriterBuilder):
    """Builder of ``NpyOutputWriter`` (the interface of ZarrOutputBuilder, output/_zarr_writer.py:93-223, with
    a directory in place of the zarr store)."""

    def __init__(self, name: str, directory: str | os.PathLike, *, time_name: str = "time",
                 overwrite: bool = False) -> None:
        self._name = name
        self._dir = Path(directory)
        self._time_name = time_name
        self._overwrite = overwrite
        self._outputs: dict[str, Output] = {}

    @property
    def name(self) -> str:
        return self._name

    @property
    def outputs(self) -> Mapping[str, Output]:
        return types.MappingProxyType(dict(self._outputs))

    def add_output(self, *outputs: Output, **kwargs) -> None:
        for output in outputs:
            if output.name in self._outputs:
                raise KeyError(f"Output variable with name '{output.name}' already exists.")
            self._outputs[output.name] = output

    def remove_output(self, name: str) -> None:
        if name not in self._outputs:
            raise KeyError(f"Output variable '{name}' does not exist.")
        del self._outputs[name]

    def build(self, nparticles: int, time_type: np.dtype = np.dtype(np.float64)) -> NpyOutputWriter:
        self._dir.mkdir(parents=True, exist_ok=True)
        names = [self._time_name] + list(self._outputs)
        for n in names:
            if (self._dir / f"{n}.npy").exists() and not self._overwrite:
                raise FileExistsError(f"{self._dir / (n + '.npy')} exists (overwrite=False)")
        return NpyOutputWriter(self._name, self._dir, self._time_name, np.dtype(time_type), self._outputs, nparticles)


__all__ = [
    "AbstractOutputWriter",
    "AbstractOutputWriterBuilder",
    "NpyOutputBuilder",
    "NpyOutputWriter",
    "Output",
    "linearly_interpolate_fields",
]
