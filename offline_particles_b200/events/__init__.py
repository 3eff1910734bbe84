"""Simulation events and their schedulers (events/ of the reference, host-side control).

An ``Event`` is a function of the simulation state plus particle kernels that
the simulation launches before calling it.  Schedulers fire events every N
iterations or every dt of simulated time, as events/_schedulers.py:13-140 of
the reference does.
"""

from __future__ import annotations

import dataclasses
from typing import Callable, Iterable

import numpy as np


@dataclasses.dataclass(frozen=True)
class SimulationState:
    time: object
    dt: object
    tidx: np.float64
    iteration: int
    particles: object


type EventFunction = Callable[[SimulationState], None]


class Event:
    """``Event(name, func, *kernels)`` (events/_events.py:26-52).  ``deferrable=True`` declares that the
    event's kernels read only the particles' status and indices and write only fields of their own, and
    that ``func`` reads only those fields and the state's time: such an event may fire after a fused
    launch on the particle state recorded at its step instead of ending the launch there."""

    def __init__(self, name: str, func: EventFunction, *kernels, deferrable: bool = False) -> None:
        self._name = name
        self._func = func
        self._kernels = kernels
        self.deferrable = bool(deferrable)

    def __call__(self, state: SimulationState) -> None:
        self._func(state)

    @property
    def name(self) -> str:
        return self._name

    @property
    def kernels(self) -> tuple:
        return self._kernels


class IterationScheduler:
    """Fires events every N iterations."""

    def __init__(self) -> None:
        self._next: int | None = None
        self._events: dict[int, list[tuple[int, Event]]] = {}

    def _schedule_event(self, iteration: int, N: int, event: Event) -> None:
        self._events.setdefault(iteration, []).append((N, event))

    @property
    def next(self) -> int | None:
        return self._next

    @property
    def events(self) -> Iterable[Event]:
        for lst in self._events.values():
            for _, event in lst:
                yield event

    def register_event(self, first: int, n: int, event: Event) -> None:
        self._schedule_event(first, n, event)
        self.set_next()

    def copy(self) -> "IterationScheduler":
        """A scheduler in the same state (the same events), to look ahead without firing."""
        c = IterationScheduler()
        c._events = {k: list(v) for k, v in self._events.items()}
        c._next = self._next
        return c

    def set_next(self) -> None:
        self._next = min(self._events) if self._events else None

    def __call__(self, iteration: int) -> list[Event]:
        fired: list[Event] = []
        while self._next is not None and self._next <= iteration:
            for N, event in self._events.pop(self._next, []):
                fired.append(event)
                self._schedule_event(self._next + N, N, event)
            self.set_next()
        return fired


class TimeScheduler:
    """Fires events every dt of simulated time."""

    def __init__(self, *, forward: bool = True) -> None:
        self._forward = forward
        self._next_time = None
        self._events: dict[object, list[tuple[object, Event]]] = {}

    def _schedule_event(self, time, dt, event: Event) -> None:
        self._events.setdefault(time, []).append((dt, event))

    @property
    def next_time(self):
        return self._next_time

    @property
    def events(self) -> Iterable[Event]:
        for lst in self._events.values():
            for _, event in lst:
                yield event

    def register_event(self, first, dt, event: Event) -> None:
        self._schedule_event(first, dt, event)
        self.set_next()

    def copy(self) -> "TimeScheduler":
        """A scheduler in the same state (the same events), to look ahead without firing."""
        c = TimeScheduler(forward=self._forward)
        c._events = {k: list(v) for k, v in self._events.items()}
        c._next_time = self._next_time
        return c

    def set_next(self) -> None:
        if not self._events:
            self._next_time = None
        elif self._forward:
            self._next_time = min(self._events)
        else:
            self._next_time = max(self._events)

    def __call__(self, time) -> list[Event]:
        fired: list[Event] = []
        while (nt := self._next_time) is not None and (nt <= time if self._forward else nt >= time):
            for dt, event in self._events.pop(nt, []):
                fired.append(event)
                self._schedule_event(nt + dt, dt, event)
            self.set_next()
        return fired


__all__ = ["Event", "SimulationState", "IterationScheduler", "TimeScheduler"]
