"""The learned scheduler's gate: a use of the cost model is switched on only when the model
beats a constant on held-out rays (R^2 > 0) and, when a measured speedup over the coherent
order is given, that speedup is above 1; otherwise the coherent order runs."""
from ever_b200.scheduler import Gate


def test_gate_needs_positive_heldout_r2():
    g = Gate(r2_events=-0.22, r2_depth=-0.01)
    assert not g.bins and not g.depth
    g = Gate(r2_events=0.0, r2_depth=0.3)
    assert not g.bins and g.depth


def test_gate_needs_a_measured_gain_when_one_is_given():
    g = Gate(r2_events=0.4, r2_depth=0.05, speedup_bins=0.94, speedup_depth=1.15)
    assert not g.bins and g.depth
    g = Gate(r2_events=0.4, r2_depth=0.05, speedup_bins=1.02, speedup_depth=0.99)
    assert g.bins and not g.depth
