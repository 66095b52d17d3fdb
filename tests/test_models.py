"""Generic robot descriptions (gato_b200.models): seeded chains and URDF
serial chains, their round trip, and their dynamics in the oracle."""
import math

import numpy as np
import pytest


def _fields(m):
    return (m.nq, [list(r) for r in m.joint_xyz], [list(r) for r in m.joint_rpy],
            [[list(b) for b in l] for l in m.link_inertial], list(m.q_limit), list(m.qd_limit),
            list(m.u_limit), m.limit_margin, m.gravity, m.barrier_style)


@pytest.mark.parametrize("nq,seed", [(7, 0), (6, 3)])
def test_seeded_chain_urdf_round_trip(nq, seed):
    from gato_b200 import models
    m = models.seeded_chain(nq, seed)
    back = models.from_urdf(models.to_urdf(m))
    a, b = _fields(m), _fields(back)
    assert a[0] == b[0]
    for x, y in zip(a[1:7], b[1:7]):
        np.testing.assert_allclose(np.array(x, float), np.array(y, float), rtol=1e-12, atol=1e-15)


def test_urdf_fixed_tail_is_merged_into_last_link():
    from gato_b200 import models
    m = models.seeded_chain(7, 1)
    text = models.to_urdf(m).replace("</robot>", (
        '  <link name="tip"><inertial><origin xyz="0 0 0.02" rpy="0 0 0"/><mass value="0.5"/>'
        '<inertia ixx="0.001" ixy="0" ixz="0" iyy="0.001" iyz="0" izz="0.002"/></inertial></link>\n'
        '  <joint name="tipj" type="fixed"><parent link="l6"/><child link="tip"/>'
        '<origin xyz="0 0 0.1" rpy="0 0 0"/></joint>\n</robot>'))
    t = models.from_urdf(text)
    body = [t.link_inertial[6][1][k] for k in range(10)]
    np.testing.assert_allclose(body[:4], [0.5, 0, 0, 0.12], atol=1e-12)
    np.testing.assert_allclose(body[4:], [0.001, 0, 0, 0.001, 0, 0.002], atol=1e-12)


def test_urdf_rejects_unsupported_chains():
    from gato_b200 import models
    m = models.seeded_chain(7, 2)
    with pytest.raises(ValueError):
        models.from_urdf(models.to_urdf(m).replace('<axis xyz="0 0 1"/>', '<axis xyz="1 0 0"/>', 1))
    six = models.to_urdf(models.seeded_chain(6, 2))
    five = six.replace('type="revolute"><parent link="l4"/>', 'type="fixed"><parent link="l4"/>')
    with pytest.raises(ValueError):
        models.from_urdf(five)


def test_seeded_chain_oracle_derivatives_match_finite_differences(oracle_mod):
    from gato_b200 import models
    O = oracle_mod
    m = models.seeded_chain(7, 4)
    om = O.Model(O.GatoModel.from_buffer_copy(bytes(m)))
    rng = np.random.default_rng(0)
    q, qd, u = rng.uniform(-1, 1, 7), rng.normal(0, 0.3, 7), rng.normal(0, 5, 7)
    qdd, df = om.fd_grad(q, qd, u)
    h = 1e-6
    for j in range(7):
        e = np.zeros(7)
        e[j] = h
        num = (om.fd(q + e, qd, u) - om.fd(q - e, qd, u)) / (2 * h)
        np.testing.assert_allclose(df[:, j], num, rtol=1e-5, atol=1e-6)
