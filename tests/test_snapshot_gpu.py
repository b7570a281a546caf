"""Asynchronous snapshots for output writers: a snapshot taken between steps holds exactly the
state of that moment (positions bitwise as tild_get_state, densities as tild_get_density), even
while later steps run and several snapshots are in flight, and a writer thread may wait for it."""
import threading

import numpy as np
import pytest

import tild
from helpers import small_diblock

pytestmark = pytest.mark.gpu


def test_snapshots_in_flight_match_synchronous_reads():
    s = small_diblock(3, 1, nx=(16, 16, 16), box=(8.0, 8.0, 8.0), seed=51)
    M = int(np.prod(s.nx))
    frames = []
    with tild.Context(s) as c:
        c.forces()
        bufs = [(tild.HostArray((s.ns, 3)), tild.HostArray((s.ntypes, M))) for _ in range(6)]
        tickets, ref = [], []
        for k, (hx, hr) in enumerate(bufs):
            tickets.append(c.snapshot_async(hx.array, hr.array))
            ref.append((c.get_state()[0], c.density()))
            c.step(7)
        done = []
        th = threading.Thread(target=lambda: [c.snapshot_wait(t) or done.append(t) for t in tickets[-3:]])
        th.start()
        th.join()
        assert done == tickets[-3:]
        for t in tickets:
            c.snapshot_wait(t)      # older tickets: already complete
        for (hx, hr), (x, rho) in zip(bufs, ref):
            assert np.array_equal(hx.array, x)
            assert np.array_equal(hr.array, rho)
        # pageable arrays work too
        x2 = np.empty((s.ns, 3), np.float32)
        t = c.snapshot_async(x2, None)
        c.snapshot_wait(t)
        assert np.array_equal(x2, c.get_state()[0])
        with pytest.raises(tild.TildError):
            c.snapshot_wait(t + 100)   # never issued
