"""The oracle pinned against the reference's analytic known-answer test
(Figure 5: a cloth sliding on a 45 degree incline, mu = 0.1)."""
import numpy as np

from conftest import incline_closed_form, load_incline
from oracle.oracle import Oracle


def test_oracle_matches_closed_form_incline():
    s, p, P = load_incline()
    o = Oracle(s, p)
    dt = P["Timestep"]
    worst_v = worst_z = 0.0
    contacts_seen = 0
    for k in range(800):
        rep = o.step(1)
        contacts_seen = max(contacts_seen, rep.n_contacts)
        q, v = o.state()
        sp, z = incline_closed_form((k + 1) * dt)
        worst_v = max(worst_v, abs(np.linalg.norm(v.mean(0)) - sp))
        worst_z = max(worst_z, abs(q[:, 2].mean() - z))
    assert contacts_seen == 4
    # speed: the discrete scheme reproduces the closed form to round-off
    assert worst_v < 1e-9, worst_v
    # height: first-order time integration lags by O(a * dt * t)
    assert worst_z < 2e-3, worst_z
