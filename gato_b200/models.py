"""Robot models for the solver: the built-in plants, seeded serial chains,
and serial revolute chains read from URDF.

The reference hard-codes each plant's spatial transforms and inertias in
GRiD-generated headers (gato/dynamics/iiwa14/iiwa14_grid.cuh init_XImats,
1209-2000; indy7_grid.cuh likewise).  Here a robot is the plain description
`gato_model_t` (include/gato_b200.h): per joint the origin (xyz, rpy) of its
frame in the parent frame, rotation about the local z axis, and per link up
to two rigid bodies (mass, centre of mass, inertia about the centre of mass in
the link frame); the library derives the transforms and spatial inertias from
it on the host.  Any 6- or 7-joint serial revolute chain can be solved.
"""
import math
import xml.etree.ElementTree as ET

import numpy as np

from . import _lib as L


def builtin(plant):
    """The reference's iiwa14 or indy7 (tables of gato_b200/csrc/plant_tables.h)."""
    return L.builtin_model(plant)


def seeded_chain(nq=7, seed=0, mass=(1.0, 4.0), length=(0.1, 0.4), width=0.08,
                 q_limit=2.9, qd_limit=2.0, u_limit=150.0):
    """A random serial revolute chain: link i is a uniform-density box
    width x width x l_i with l_i ~ U[length] and mass ~ U[mass], its centre
    of mass half-way along the link's z axis; joint i+1 sits at the end of
    link i, turned by +-pi/2 about x so that consecutive axes alternate
    (a non-planar arm)."""
    if nq not in (6, 7):
        raise ValueError("the solver is built for 6 or 7 joints")
    rng = np.random.default_rng(seed)
    m = L.GatoModel()
    m.nq = nq
    lengths = rng.uniform(*length, nq)
    masses = rng.uniform(*mass, nq)
    for i in range(nq):
        xyz = (0.0, 0.0, 0.1 if i == 0 else float(lengths[i - 1]))
        rpy = (0.0 if i == 0 else (math.pi / 2 if i % 2 else -math.pi / 2), 0.0, 0.0)
        for a in range(3):
            m.joint_xyz[i][a] = xyz[a]
            m.joint_rpy[i][a] = rpy[a]
        li, mi = float(lengths[i]), float(masses[i])
        ixx = mi / 12.0 * (width ** 2 + li ** 2)
        izz = mi / 12.0 * (2 * width ** 2)
        body = (mi, 0.0, 0.0, li / 2, ixx, 0.0, 0.0, ixx, 0.0, izz)
        for k in range(10):
            m.link_inertial[i][0][k] = body[k]
            m.link_inertial[i][1][k] = 0.0
        m.q_limit[i] = q_limit
        m.qd_limit[i] = qd_limit
        m.u_limit[i] = u_limit
    m.limit_margin = -0.1
    m.gravity = 9.81
    m.barrier_style = 0
    return m


def _floats(s, n=3):
    v = [float(x) for x in (s or "").split()]
    return v + [0.0] * (n - len(v))


def _rpy_matrix(r, p, y):
    cr, sr, cp, sp, cy, sy = (math.cos(r), math.sin(r), math.cos(p), math.sin(p),
                              math.cos(y), math.sin(y))
    rx = np.array([[1, 0, 0], [0, cr, -sr], [0, sr, cr]])
    ry = np.array([[cp, 0, sp], [0, 1, 0], [-sp, 0, cp]])
    rz = np.array([[cy, -sy, 0], [sy, cy, 0], [0, 0, 1]])
    return rz @ ry @ rx


def _inertial(link):
    """(mass, com [3], inertia 3x3 about the com in the link frame) of a URDF
    <link>, or None."""
    el = link.find("inertial")
    if el is None:
        return None
    mass = float(el.find("mass").get("value"))
    org = el.find("origin")
    com = np.array(_floats(org.get("xyz") if org is not None else None))
    rot = _rpy_matrix(*_floats(org.get("rpy") if org is not None else None))
    ie = el.find("inertia")
    g = lambda k: float(ie.get(k, 0.0))
    I = np.array([[g("ixx"), g("ixy"), g("ixz")], [g("ixy"), g("iyy"), g("iyz")],
                  [g("ixz"), g("iyz"), g("izz")]])
    return mass, com, rot @ I @ rot.T


def from_urdf(urdf, q_margin=-0.1, gravity=9.81, barrier_style=0):
    """gato_model_t of the serial revolute chain in a URDF (a path or the XML
    text).  Joints are taken from the root down; every revolute/continuous
    joint must turn about its z axis.  Links hanging on fixed joints below
    the last moving joint are merged into the last link as its second body
    (as the reference's iiwa14 merges its `contact` link); the end effector
    is the origin of the last moving joint's frame."""
    text = urdf
    if not urdf.lstrip().startswith("<"):
        with open(urdf) as f:
            text = f.read()
    root = ET.fromstring(text)
    links = {l.get("name"): l for l in root.findall("link")}
    joints = root.findall("joint")
    by_parent = {}
    for j in joints:
        by_parent.setdefault(j.find("parent").get("link"), []).append(j)
    children = {j.find("child").get("link") for j in joints}
    roots = [n for n in links if n not in children]
    if len(roots) != 1:
        raise ValueError("expected one root link")
    moving, fixed_tail = [], []
    cur = roots[0]
    while cur in by_parent:
        js = by_parent[cur]
        if len(js) != 1:
            raise ValueError(f"link {cur!r} branches: only serial chains are supported")
        j = js[0]
        kind = j.get("type")
        if kind in ("revolute", "continuous"):
            if fixed_tail:
                raise ValueError("a fixed joint between moving joints is not supported")
            axis = _floats(j.find("axis").get("xyz") if j.find("axis") is not None else "1 0 0")
            if not np.allclose(axis, [0, 0, 1]):
                raise ValueError(f"joint {j.get('name')!r}: only rotation about z is supported")
            moving.append(j)
        elif kind == "fixed":
            if moving:
                fixed_tail.append(j)
        else:
            raise ValueError(f"joint type {kind!r} is not supported")
        cur = j.find("child").get("link")
    nq = len(moving)
    if nq not in (6, 7):
        raise ValueError(f"{nq} moving joints: the solver is built for 6 or 7")
    m = L.GatoModel()
    m.nq = nq
    for i, j in enumerate(moving):
        org = j.find("origin")
        xyz = _floats(org.get("xyz") if org is not None else None)
        rpy = _floats(org.get("rpy") if org is not None else None)
        for a in range(3):
            m.joint_xyz[i][a] = xyz[a]
            m.joint_rpy[i][a] = rpy[a]
        lim = j.find("limit")
        lo = float(lim.get("lower", -math.pi)) if lim is not None else -math.pi
        hi = float(lim.get("upper", math.pi)) if lim is not None else math.pi
        m.q_limit[i] = max(abs(lo), abs(hi))
        m.qd_limit[i] = float(lim.get("velocity", 10.0)) if lim is not None else 10.0
        m.u_limit[i] = float(lim.get("effort", 100.0)) if lim is not None else 100.0
        bodies = []
        ine = _inertial(links[j.find("child").get("link")])
        if ine is not None:
            bodies.append(ine)
        if i == nq - 1:
            # fixed links below the last joint, expressed in its frame
            R, p = np.eye(3), np.zeros(3)
            for f in fixed_tail:
                org = f.find("origin")
                Rf = _rpy_matrix(*_floats(org.get("rpy") if org is not None else None))
                pf = np.array(_floats(org.get("xyz") if org is not None else None))
                p, R = p + R @ pf, R @ Rf
                ine = _inertial(links[f.find("child").get("link")])
                if ine is not None:
                    mass, com, I = ine
                    bodies.append((mass, p + R @ com, R @ I @ R.T))
        if len(bodies) > 2:
            raise ValueError("at most two bodies per link")
        for bi in range(2):
            vals = [0.0] * 10
            if bi < len(bodies):
                mass, com, I = bodies[bi]
                vals = [mass, *com, I[0, 0], I[0, 1], I[0, 2], I[1, 1], I[1, 2], I[2, 2]]
            for k in range(10):
                m.link_inertial[i][bi][k] = float(vals[k])
    m.limit_margin = q_margin
    m.gravity = gravity
    m.barrier_style = barrier_style
    return m


def to_urdf(m, name="chain"):
    """URDF text of a model (inverse of from_urdf for single-body links)."""
    out = [f'<robot name="{name}">', '  <link name="base"/>']
    for i in range(m.nq):
        b = [m.link_inertial[i][0][k] for k in range(10)]
        out.append(f'  <link name="l{i}"><inertial><origin xyz="{b[1]} {b[2]} {b[3]}" '
                   f'rpy="0 0 0"/><mass value="{b[0]}"/><inertia ixx="{b[4]}" ixy="{b[5]}" '
                   f'ixz="{b[6]}" iyy="{b[7]}" iyz="{b[8]}" izz="{b[9]}"/></inertial></link>')
        parent = "base" if i == 0 else f"l{i - 1}"
        xyz = " ".join(str(m.joint_xyz[i][a]) for a in range(3))
        rpy = " ".join(str(m.joint_rpy[i][a]) for a in range(3))
        out.append(f'  <joint name="j{i}" type="revolute"><parent link="{parent}"/>'
                   f'<child link="l{i}"/><origin xyz="{xyz}" rpy="{rpy}"/><axis xyz="0 0 1"/>'
                   f'<limit lower="{-m.q_limit[i]}" upper="{m.q_limit[i]}" '
                   f'velocity="{m.qd_limit[i]}" effort="{m.u_limit[i]}"/></joint>')
    out.append("</robot>")
    return "\n".join(out)
