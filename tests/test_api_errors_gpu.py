"""Error behaviour of the C ABI on the GPU: a call that fails returns its status and leaves the
context usable, with the state it had before the call (the reference's die() would end the
process instead, die.cu:3-6)."""
import numpy as np
import pytest

import tild
from helpers import small_diblock

pytestmark = pytest.mark.gpu


def test_non_finite_positions_are_rejected_before_the_state_changes():
    s = small_diblock(3, 1)
    with tild.Context(s) as c:
        c.step(3)
        before = c.get_state()
        bad = before[0].copy()
        bad[17, 1] = np.nan
        with pytest.raises(tild.TildError) as e:
            c.set_state(bad)
        assert e.value.status == tild.ERR_NAN
        after = c.get_state()
        for a, b in zip(before, after):
            assert np.array_equal(a, b)
        bad[17, 1] = np.inf
        with pytest.raises(tild.TildError):
            c.set_state(bad)
        c.step(2)                                # still steps from the kept state
        assert np.isfinite(c.get_state()[0]).all()
