"""GPU parity of the batched device time step (include/winds_wake.h) against
the FP64 step oracle (oracle/wake_ref.py), two uneven cases per batch."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import per_target_rel

pytestmark = pytest.mark.gpu


def _cases(synth):
    a = synth.make_wake_case(synth.RotorCase(nst=9, nsteps=14, dpsi_deg=8.0, seed=21, jitter=0.0),
                             nsteps=10, jitter=0.02)
    b = synth.make_wake_case(synth.RotorCase(nst=6, nb=2, nsteps=22, dpsi_deg=6.0, U=8.0,
                                             yaw_deg=20.0, shear=0.2, seed=22), nsteps=10, jitter=0.02)
    return [a, b]


def _refs(wake_ref, cases, **kw):
    return [wake_ref.WakeRef(wake_ref.WakeCaseRef(**{k: c[k] for k in wake_ref.WakeCaseRef.__dataclass_fields__}),
                             **kw) for c in cases]


@pytest.mark.parametrize("integ", ["fe", "ab2", "ab4", "pcc"])
@pytest.mark.parametrize("prec", ["f64", "f32c"])
def test_device_step_matches_oracle(wb, synth, integ, prec):
    import wake_ref
    wake = __import__("importlib").import_module("winds-master_b200.wake")
    cases = _cases(synth)
    batch = wake.WakeBatch(cases, integrator=integ, precision=prec)
    refs = _refs(wake_ref, cases, integrator=integ)
    tol_u = 1e-10 if prec == "f64" else 1e-5
    for step in range(5):
        batch.step(1)
        for k, r in enumerate(refs):
            r.step()
            st = batch.state(k)
            np.testing.assert_allclose(st["shed"], r.shed, rtol=0, atol=1e-12)
            np.testing.assert_allclose(st["trail"], r.trail, rtol=0, atol=1e-12)
            # stretched cores follow the node positions, which carry the path's velocity error
            tol_rc = 1e-12 if prec == "f64" else 1e-6
            np.testing.assert_allclose(st["rc_shed"], r.rcs, rtol=tol_rc)
            np.testing.assert_allclose(st["rc_trail"], r.rct, rtol=tol_rc)
            assert per_target_rel(st["uind"], r.uind) < tol_u, (step, k)
            # positions: the step's displacement carries the velocity error
            disp = np.abs(r.dom[:, :, 2:] - st["dom"][:, :, 2:]).max()
            scale = cases[k]["dt"] * np.abs(r.uind).max() * (step + 1)
            assert disp <= (1e-9 if prec == "f64" else 3e-5) * max(scale, 1.0), (step, k, disp)


def test_graph_replay_is_bit_identical(wb, synth):
    wake = __import__("importlib").import_module("winds-master_b200.wake")
    cases = _cases(synth)
    a = wake.WakeBatch(cases, integrator="pcc")
    b = wake.WakeBatch(cases, integrator="pcc")
    a.step(4, graph=False)
    b.step(4, graph=True)
    for k in range(2):
        sa, sb = a.state(k), b.state(k)
        for key in ("dom", "uind", "shed", "trail"):
            np.testing.assert_array_equal(sa[key], sb[key])


def test_bound_update_enters_next_step(wb, synth):
    """A new bound circulation (as a Kutta-Joukowski iteration leaves it)
    shapes the next step's trailing and shed columns (WInDS.m:131-140)."""
    import wake_ref
    wake = __import__("importlib").import_module("winds-master_b200.wake")
    cases = _cases(synth)
    batch = wake.WakeBatch(cases, integrator="pcc", precision="f64")
    refs = _refs(wake_ref, cases, integrator="pcc")
    batch.step(2)
    for r in refs:
        r.step(), r.step()
    nb = 1.3 * refs[0].bound
    batch.set_bound(0, nb)
    refs[0].bound = nb
    batch.step(1)
    refs[0].step()
    st = batch.state(0)
    np.testing.assert_allclose(st["shed"], refs[0].shed, rtol=0, atol=1e-12)
    assert per_target_rel(st["uind"], refs[0].uind) < 1e-10


def test_kinematics_limit_is_enforced(wb, synth):
    wake = __import__("importlib").import_module("winds-master_b200.wake")
    batch = wake.WakeBatch(_cases(synth), integrator="fe")
    with pytest.raises(wb.WindsError):
        batch.step(20)


def test_first_step_autotunes_the_batch_tiling(wb, synth):
    """An FP32c batch whose size has no cached tiling times the candidates on
    its first step and caches the fastest for its size bucket."""
    wake = __import__("importlib").import_module("winds-master_b200.wake")
    cases = [synth.make_wake_case(rc, nsteps=4) for rc in synth.batch_cases(5, seed=77, steps_range=(300, 400))]
    nodes = sum(c["nst"] * c["na"] * c["nb"] for c in cases)
    fil = sum(((c["nst"] - 1) * c["na"] + c["nst"] * (c["na"] - 1)) * c["nb"] for c in cases)
    b = wake.WakeBatch(cases, integrator="fe", precision="f32c")
    b.step(1)
    T, KF, waves = wb.get_tuning(wb.bs.CORE_VATISTAS, nodes, fil)
    assert T in (3, 4) and KF in (32, 64) and waves in (32.0, 64.0)
    b.close()


def test_sharded_run_device_stepper_matches_the_batch(wb, synth):
    """sharding.ShardedRun on one rank with the device stepper gives the
    batch's own thrust, torque, power and iteration counts every step."""
    import importlib
    sh = importlib.import_module("winds-master_b200.sharding")
    wake = importlib.import_module("winds-master_b200.wake")
    rcs = synth.batch_cases(3, seed=8, steps_range=(20, 40), nodes_range=(9, 13))
    cases = [synth.make_wake_case(rc, nsteps=4) for rc in rcs]
    kjs = [synth.make_kj_case(rc, nsteps=4, t0=c["t0"]) for rc, c in zip(rcs, cases)]
    kp = dict(relax=0.3, tol=1e-6, maxiter=100)
    run = sh.ShardedRun(cases, kjs, rank=0, world=1, integrator="pcc", precision="f32c", kj_params=kp)
    b = wake.WakeBatch(cases, integrator="pcc", precision="f32c")
    b.set_kj(kjs, **kp)
    for _ in range(2):
        got = run.step(1, graph=True)
        b.step(1, graph=True)
        T, Q, P = b.loads()
        want = np.stack([T, Q, P, b.kj_stats()[0].astype(np.float64)], 1)
        np.testing.assert_array_equal(got, want)
    run.close()
    b.close()
