"""FP64 oracle of the rotor loads (test infrastructure).

Restates ``postproc/perform.m:18-62`` for one case and one step:
  * blade-frame velocity to the rotor frame, removing twist and pitch
    (``:20-26``): ``velX = -DCMRot(vblade, [-90, twist, pitch], 'zzz')``; the
    three rotations share the z axis, so ``velX = -Rz(twist + pitch - 90) vblade``
    with ``Rz(t) = [[cos t, -sin t, 0], [sin t, cos t, 0], [0, 0, 1]]``
    (``core/DCMRot.m:27-45,73-75``);
  * local tip-speed ratio ``velX2 / velX1`` (``:27``), inflow angle
    ``phi = aoa - (pitch + twist)`` (``:35``);
  * ``a/a' = TSR / tan(phi)``, ``a`` and ``a'`` (``:41-43``);
  * normal / tangential coefficients (``:45-46``), spanwise thrust, torque and
    power (``:48-55``), rotor totals summed over stations and blades (``:59-61``).
"""
from __future__ import annotations

import numpy as np


def rz(t_deg):
    t = np.radians(t_deg)
    c, s = np.cos(t), np.sin(t)
    R = np.zeros(np.shape(t) + (3, 3))
    R[..., 0, 0], R[..., 0, 1], R[..., 1, 0], R[..., 1, 1], R[..., 2, 2] = c, -s, s, c, 1.0
    return R


def loads(cl, cd, aoa, vblade, theta_deg, chord, r, dr, rpm, rho):
    """cl, cd, aoa [ns, nb] (aoa in deg); vblade [ns, 3, nb]; theta_deg [ns]
    or [ns, nb] (twist + blade pitch, perform.m:22-33 per blade); chord, r, dr
    [ns]; rpm scalar. Returns T, Q, P and the spanwise dT [ns, nb]."""
    th = np.asarray(theta_deg, dtype=np.float64)
    if th.ndim == 1:
        th = np.repeat(th[:, None], np.shape(aoa)[1], axis=1)
    R = rz(th - 90.0)                                          # [ns, nb, 3, 3]
    velX = -np.einsum("sbij,sjb->sib", R, vblade)              # [ns, 3, nb]
    v1, v2 = velX[:, 0], velX[:, 1]
    tsr = v2 / v1
    phi = aoa - th
    tp = np.tan(np.radians(phi))
    aap = tsr / tp
    a = aap * (v1 - tp * v2) / (aap * v1 + tp * v2)
    ap = a / aap
    cz = cl * np.cos(np.radians(phi)) + cd * np.sin(np.radians(phi))
    cx = cl * np.sin(np.radians(phi)) - cd * np.cos(np.radians(phi))
    w2 = (v1 * (1 - a)) ** 2 + (v2 * (1 + ap)) ** 2
    c = np.asarray(chord)[:, None]
    dT = 0.5 * rho * c * cz * w2 * np.asarray(dr)[:, None]
    dQ = 0.5 * rho * c * cx * w2 * np.asarray(r)[:, None] * np.asarray(dr)[:, None]
    dP = (np.pi / 30.0) * rpm * dQ
    return float(dT.sum()), float(dQ.sum()), float(dP.sum()), dT
