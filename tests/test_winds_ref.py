"""CPU tests of the literal driver-loop oracle (oracle/winds_ref.py): the
growing cell arrays of core/initials.m and WInDS.m, Kelvin's theorem in the
bookkeeping, the integrators' time-index switches, and its agreement with the
truncated-wake step oracle (oracle/wake_ref.py) on the step they share."""
from __future__ import annotations

import numpy as np
import pytest

from run_inputs import cl0_geometric, nrel_series, oracle_run


@pytest.fixture(scope="module")
def run_inputs():
    import kin_ref
    m, ser = nrel_series(nsteps=8)
    kin = kin_ref.kinematics(ser)
    return m, ser, kin, cl0_geometric(m, ser, kin)


def test_initial_state_is_two_columns(run_inputs):
    """core/initials.m:84-86,124-131: wake.domain{1} holds the quarter-chord
    and trailing-edge nodes, shed{1} = [G, -G], trail{1} = diff([0; G; 0]);
    fe then fills the third column of wake.domain{2}."""
    m, ser, kin, cl0 = run_inputs
    r = oracle_run(m, ser, kin, cl0)
    assert r.domain[1].shape[2] == 2 and r.domain[2].shape[2] == 3
    G = r.shed[1][:, 0]
    np.testing.assert_allclose(r.shed[1][:, 1], -G, rtol=0, atol=1e-12 * np.abs(G).max())
    np.testing.assert_array_equal(r.trail[1][:, 0], np.diff(np.concatenate([np.zeros((1, 3)), G,
                                                                           np.zeros((1, 3))]), axis=0))
    np.testing.assert_allclose(r.domain[2][:, :, 2], r.domain[1][:, :, 1] + r.dt * r.vel[1][:, :, 1],
                               rtol=0, atol=1e-12)
    # wake.r0 per step from TSR and |U| (initials.m:134-135) changes with the gust
    assert np.ptp(r.r0) > 0


@pytest.mark.parametrize("integ", ["fe", "ab2", "ab4", "pcc"])
def test_wake_grows_one_column_per_step(run_inputs, integ):
    m, ser, kin, cl0 = run_inputs
    r = oracle_run(m, ser, kin, cl0, integ=integ, tol=1e-6)
    for _ in range(4):
        p = r.step()
        assert r.domain[p].shape[2] == p + 1 and r.shed[p].shape[1] == p + 1
        assert r.trail[p].shape[1] == p
        # Kelvin: every trailing column sums to zero over the span
        np.testing.assert_allclose(r.trail[p].sum(axis=0), 0.0, atol=1e-10)
        assert 1 <= r.ctj <= 30
        assert np.isfinite(r.T) and np.isfinite(r.P) and r.T > 0


def test_pcc_corrector_starts_at_time_index_three(run_inputs):
    """pcc.m:40: at time <= 2 the predictor stands (domain{p+1} = fe); from
    time 3 on the corrector changes it."""
    m, ser, kin, cl0 = run_inputs
    a = oracle_run(m, ser, kin, cl0, integ="pcc", tol=1e-6)
    b = oracle_run(m, ser, kin, cl0, integ="fe", tol=1e-6)
    a.step()  # p = 2
    b.step()
    np.testing.assert_array_equal(a.domain[3], b.domain[3])
    a.step()  # p = 3: corrector
    b.step()
    assert np.abs(a.domain[4][:, :, 2:] - b.domain[4][:, :, 2:]).max() > 1e-9


def test_bookkeeping_agrees_with_truncated_step_oracle(run_inputs):
    """WInDS.m:131-140 keeps every trailing column (trail{p}(:,2:end) =
    trail{p-1}); the truncated-wake oracle (oracle/wake_ref.py) drops its
    last one. Given one spare zero column, the truncated bookkeeping must
    reproduce the growing one exactly, and the induced velocity of the two
    oracles' evaluation paths on the same state must agree."""
    import wake_ref
    m, ser, kin, cl0 = run_inputs
    r = oracle_run(m, ser, kin, cl0, integ="fe", tol=1e-6)
    for _ in range(3):
        r.step()
    p = r.p + 1
    r.bookkeeping(p)
    r.vcore(p)
    prev = r.trail[p - 1]
    spare = np.concatenate([prev, np.zeros((prev.shape[0], 1, prev.shape[2]))], axis=1)
    shed, trail = wake_ref.bookkeeping(r.shed[p - 1][:, 0, :], spare)
    np.testing.assert_array_equal(trail, r.trail[p])
    np.testing.assert_array_equal(shed, r.shed[p])
    u = wake_ref.induced(r.domain[p], shed, trail, r.rce_s[p], r.rce_t[p], 1e-4, 1000.0)
    np.testing.assert_array_equal(u, r.induced(p))
