"""The order in which snapshot rings issue their uploads onto a device's shared copy stream
(fields.TicketOrder): host logic, no GPU."""

from __future__ import annotations

import threading
import time

from offline_particles_b200.fields import TicketOrder


def _run(order: TicketOrder, tickets_and_delays, limit=None):
    """Each (ticket, delay) in its own thread: sleep, wait for the turn, record the issue, release."""
    issued, results = [], {}
    lock = threading.Lock()

    def work(t, delay):
        time.sleep(delay)
        ok = order.wait_turn(t, limit)
        with lock:
            issued.append(t)
            results[t] = ok
        order.release(t)

    threads = [threading.Thread(target=work, args=td) for td in tickets_and_delays]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    return issued, results


def test_issue_follows_ticket_order_whatever_the_threads_do():
    order = TicketOrder(limit=5.0)
    tickets = [order.ticket() for _ in range(8)]
    assert tickets == list(range(8))
    # later tickets are ready first: they still issue in ticket order
    issued, results = _run(order, [(t, 0.02 * (8 - t)) for t in tickets])
    assert issued == tickets and all(results.values())


def test_a_stuck_ticket_is_passed_over_once_then_ignored():
    order = TicketOrder(limit=5.0)
    stuck, a, b = order.ticket(), order.ticket(), order.ticket()
    t0 = time.perf_counter()
    # b starts waiting later, so a's wait is the first to run out (both waits are 0.2 s)
    issued, results = _run(order, [(a, 0.0), (b, 0.05)], limit=0.2)
    took = time.perf_counter() - t0
    assert issued == [a, b]
    assert results[a] is False and results[b] is True  # only the first waiter waits for the stuck one
    assert 0.15 < took < 2.0
    order.release(stuck)  # the stuck upload finally issues: nothing changes
    c = order.ticket()
    assert order.wait_turn(c, 0.5) is True


def test_release_without_waiting_keeps_the_order_moving():
    order = TicketOrder()
    t = [order.ticket() for _ in range(3)]
    order.release(t[1])
    assert order.issued_below == 0
    order.release(t[0])
    assert order.issued_below == 2
    order.release(t[2])
    assert order.issued_below == 3 and not order.done


class _FakeField:
    """What _prefetch_after touches on a TimeDependentField, recording the order of prefetches."""

    def __init__(self, name, log, ring_size=8, streamed=True):
        self.name, self.log, self.ring_size, self.streamed = name, log, ring_size, streamed

    def mark_used(self, ks):
        pass

    def prefetch(self, k, keep):
        assert k in keep
        self.log.append((k, self.name))


def test_prefetch_after_a_launch_goes_snapshot_by_snapshot():
    from offline_particles_b200.timesteppers import _prefetch_after

    log = []
    td = {n: _FakeField(n, log) for n in ("u", "v", "w", "zeta")}
    _prefetch_after(td, [0, 1, 2], limit=5)
    # every field's snapshot 3 before any field's 4, and nothing past the run's horizon
    assert log == [(k, n) for k in (3, 4, 5) for n in ("u", "v", "w", "zeta")]


def test_prefetch_depth_follows_each_ring():
    from offline_particles_b200.timesteppers import _prefetch_after

    log = []
    td = {"u": _FakeField("u", log, ring_size=4), "v": _FakeField("v", log, ring_size=6),
          "zeta": _FakeField("zeta", log, streamed=False)}
    _prefetch_after(td, [0, 1, 2])
    # keep {1, 2}: a ring of 4 prefetches 2 ahead, a ring of 6 four ahead, a resident field none
    assert log == [(3, "u"), (3, "v"), (4, "u"), (4, "v"), (5, "v"), (6, "v")]
