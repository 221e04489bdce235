"""Pin the oracle's nodal update to the reference's known answers in
tests/nodes/node_test.cc (3D node, Nphase 0, dt = 0.1):

* "Check compute acceleration and velocity" (node_test.cc:1573-1640):
  mass 100, internal force 10 i, external force 5 i, then a velocity
  constraint v_x = 10.5, then Cundall damping 0.05;
* "Check Cartesian friction constraints" (node_test.cc:1844-1858): velocity
  0.1, acceleration 5 in every direction, friction (dir 2, sign 2, mu 0.3).
"""
import numpy as np

from oracle.oracle import Oracle
from tests.conftest import catch_approx

EPS = 1e-7


def _close(a, b):
    return all(catch_approx(x, y, EPS) for x, y in zip(np.ravel(a), np.ravel(b)))


def _one_cell(damping=0.0):
    o = Oracle(3, dt=0.1, damping_factor=damping)
    X = np.array([[0, 0, 0], [2, 0, 0], [2, 2, 0], [0, 2, 0],
                  [0, 0, 2], [2, 0, 2], [2, 2, 2], [0, 2, 2]], dtype=float)
    o.set_mesh(X, np.arange(8)[None, :])
    return o


def _node_table(mass, fint=(0, 0, 0), fext=(0, 0, 0), vel=(0, 0, 0), acc=(0, 0, 0)):
    t = np.zeros((8, 17))
    t[0, 0] = mass
    t[0, 4:7] = fext
    t[0, 7:10] = fint
    t[0, 10:13] = vel
    t[0, 13:16] = acc
    t[0, 16] = 1.0
    return t


def test_compute_acceleration_velocity_and_cundall():
    o = _one_cell()
    o.set_nodes(_node_table(100., fint=(0., 10., 20.), fext=(0., 5., 10.)))
    o.phase("node_update", dt=0.1)
    n = o.nodes(8)[0]
    force = np.array([0., 15., 30.])
    # node_test.cc:1598-1606
    assert _close(n[13:16], force / 100.)
    assert _close(n[10:13], force / 100. * 0.1)
    # node_test.cc:1608-1619: velocity constraint in x
    o.add_velocity_constraints([0], [0], [10.5])
    o.phase("node_update", dt=0.1)
    n = o.nodes(8)[0]
    assert _close(n[10:13], [10.5, 0.03, 0.06])
    assert _close(n[13:16], [0.0, 0.15, 0.3])
    # node_test.cc:1620-1627: the same node with Cundall damping 0.05
    o2 = _one_cell(damping=0.05)
    o2.add_velocity_constraints([0], [0], [10.5])
    o2.set_nodes(o.nodes(8))
    o2.phase("node_update", dt=0.1)
    n = o2.nodes(8)[0]
    assert _close(n[13:16], [0.0, 0.13322949016875, 0.28322949016875])
    # node_test.cc:1634-1639: zero mass, no update
    o2.set_nodes(_node_table(0., fint=(1., 1., 1.)))
    o2.phase("node_update", dt=0.1)
    assert _close(o2.nodes(8)[0][13:16], [0., 0., 0.])


def test_cartesian_friction_3d():
    o = _one_cell()
    o.add_friction_constraints([0], [2], [2], [0.3])
    # acceleration (5, 5, 5) from forces 500 on mass 100, velocity 0.1
    o.set_nodes(_node_table(100., fext=(500., 500., 500.), vel=(0.1, 0.1, 0.1)))
    o.phase("node_update", dt=0.1)
    n = o.nodes(8)[0]
    # node_test.cc:1852-1857
    assert _close(n[13:16], [3.939339828220179, 3.939339828220179, 5.])
