"""Host-side forward kinematics of a gato_model_t chain (numpy, FP64), for
`BSQP.ee_pos` and for building goals: the position of the last link frame
origin, the point the tracking cost follows.  Uses the same transform rules as
the CUDA library (entries below 1e-6 of the fixed joint rotations are zeroed).
"""
import numpy as np

SNAP = 1e-6


def _rpy(r, p, y):
    cr, sr, cp, sp, cy, sy = np.cos(r), np.sin(r), np.cos(p), np.sin(p), np.cos(y), np.sin(y)
    Rx = np.array([[1, 0, 0], [0, cr, -sr], [0, sr, cr]])
    Ry = np.array([[cp, 0, sp], [0, 1, 0], [-sp, 0, cp]])
    Rz = np.array([[cy, -sy, 0], [sy, cy, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def ee_position(model, q):
    """q: (..., nq) joint angles -> (..., 3) end-effector positions."""
    q = np.asarray(q, dtype=np.float64)
    nq = model.nq
    R0 = []
    P = []
    for i in range(nq):
        R = _rpy(*model.joint_rpy[i])
        R[np.abs(R) < SNAP] = 0.0
        R0.append(R)
        P.append(np.array(model.joint_xyz[i][:3]))
    flat = q.reshape(-1, nq)
    out = np.zeros((flat.shape[0], 3))
    for n, qq in enumerate(flat):
        R = np.eye(3)
        o = np.zeros(3)
        for i in range(nq):
            o = o + R @ P[i]
            c, s = np.cos(qq[i]), np.sin(qq[i])
            R = R @ R0[i] @ np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])
        out[n] = o
    return out.reshape(q.shape[:-1] + (3,))
