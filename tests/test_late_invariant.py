"""The slot arithmetic the late delivery relies on (no GPU).

The engine's ring has L = max(min_delay, max_delay) slots; a spike emitted at
step t with delay d lands in slot (t + d) mod L and is read by the update of
step t + d (NEST's slot rule, event_delivery_manager.cpp / ring_buffer.h).  An
edge of delay d >= 2 min_delay from a spike of the slice [o, o + md) arrives
at or after o + 2 md, so (1) the next slice's update never needs it and (2)
the slot it is added to is none of the slots that update reads and clears;
the slice after next waits for it.  Delays below 2 md may arrive in the next
slice, so they stay with the slice-close delivery.
"""

from hypothesis import given, settings
from hypothesis import strategies as st


@settings(max_examples=3000, deadline=None)
@given(md=st.integers(1, 16), extra=st.integers(0, 120), o_slices=st.integers(0, 10_000), lag=st.integers(0, 15),
       dfrac=st.floats(0.0, 1.0))
def test_late_edges_miss_the_next_slice(md, extra, o_slices, lag, dfrac):
    max_delay = md + extra
    L = max(md, max_delay)
    o = o_slices * md
    t = o + lag % md
    read_next = {(o + md + k) % L for k in range(md)}       # slots slice s+1 reads and clears
    if max_delay >= 2 * md:
        d = 2 * md + int(dfrac * (max_delay - 2 * md))
        assert t + d >= o + 2 * md
        assert (t + d) % L not in read_next
    # a delay below 2 md can be needed by the next slice (so it is not late)
    if max_delay >= md:
        d = md + int(dfrac * (min(max_delay, 2 * md - 1) - md))
        if d < 2 * md and t + d < o + 2 * md:
            assert (t + d) % L in read_next


@settings(max_examples=2000, deadline=None)
@given(md=st.integers(1, 16), extra=st.integers(0, 120), o_slices=st.integers(0, 10_000))
def test_late_edges_of_consecutive_slices_never_meet_an_open_read(md, extra, o_slices):
    """While the late delivery of slice s runs beside slice s+1, it writes only
    arrivals of slices >= s+2; the ring never wraps onto a slot of slice s+1
    within max_delay steps."""
    max_delay = md + extra
    if max_delay < 2 * md:
        return
    L = max(md, max_delay)
    o = o_slices * md
    read_next = {(o + md + k) % L for k in range(md)}
    for lag in range(md):
        for d in range(2 * md, max_delay + 1):
            assert (o + lag + d) % L not in read_next
