"""Pin the oracle's P2G / nodal update / strain / stress / force chain to the
reference's known answers in tests/particles/particle_test.cc (3D section
"Test particle, cell and node functions", lines 2371-2900): one hex8 cell of
side 2, one particle at (1.5, 1.5, 1.5), LinearElastic E=1e7, nu=0.3,
density 1000.  Values and line numbers are those of the reference test; the
comparison is Catch v1.12 Approx with epsilon 1e-7.
"""
import numpy as np

from oracle.oracle import Oracle
from tests.conftest import catch_approx

EPS = 1e-7


def _close(a, b, eps=EPS):
    a = np.asarray(a, dtype=float).ravel()
    b = np.asarray(b, dtype=float).ravel()
    return all(catch_approx(x, y, eps) for x, y in zip(a, b))


def _one_cell_3d(dt=0.1):
    o = Oracle(3, scheme="usf", dt=dt)
    X = np.array([[0, 0, 0], [2, 0, 0], [2, 2, 0], [0, 2, 0],
                  [0, 0, 2], [2, 0, 2], [2, 2, 2], [0, 2, 2]], dtype=float)
    o.set_mesh(X, np.arange(8)[None, :])
    o.add_material(0, "LinearElastic", {"density": 1000., "youngs_modulus": 1.0E+7,
                                        "poisson_ratio": 0.3})
    o.add_particles(np.array([[1.5, 1.5, 1.5]]), 0)
    o.initialise()
    return o


def test_particle_chain_3d():
    o = _one_cell_3d()
    p = o.get()
    # particle_test.cc:2493-2496 compute_volume -> 8; :2515 mass 8000
    assert _close(p["volume"], [8.0]) and _close(p["mass"], [8000.])
    # :2499-2503 reference location (0.5, 0.5, 0.5)
    assert _close(p["xi"][0], [0.5, 0.5, 0.5])
    o.set({"v": np.array([[0.0, 1.0, 2.0]])})
    o.phase("initialise")
    o.phase("p2g_mass_momentum")
    nodes = o.nodes(8)
    # :2569-2574 nodal mass
    assert _close(nodes[:, 0], [125., 375., 1125., 375., 375., 1125., 3375., 1125.])
    o.phase("compute_velocity")
    nodes = o.nodes(8)
    # :2580-2596 nodal momentum, :2598-2614 nodal velocity
    mom = np.array([[0, 125, 250], [0, 375, 750], [0, 1125, 2250], [0, 375, 750],
                    [0, 375, 750], [0, 1125, 2250], [0, 3375, 6750], [0, 1125, 2250]], float)
    assert _close(nodes[:, 1:4], mom)
    assert _close(nodes[:, 10:13], np.tile([0., 1., 2.], (8, 1)))
    # :2643-2668 momentum overwritten with row i scaled by (i+1)
    scale = np.arange(1, 9, dtype=float)[:, None]
    nodes[:, 1:4] = mom * scale
    o.set_nodes(nodes)
    o.phase("compute_velocity")
    nodes = o.nodes(8)
    vel = np.array([[0, i, 2 * i] for i in range(1, 9)], dtype=float)
    assert _close(nodes[:, 10:13], vel)
    # one stress-strain pass with dt = 0.1 (mpm_scheme.tcc:75-103)
    o.phase("stress_strain", dt=0.1)
    p = o.get()
    # :2676-2687 deformation gradient
    assert _close(p["F"][0], [1., 0., 0., -0.025, 1.075, 0.2, -0.05, 0.15, 1.4])
    # :2693-2700 strain after one increment
    assert _close(p["strain"][0], [0.0, 0.075, 0.4, -0.025, 0.35, -0.05])
    # :2707-2709 volume 8 -> 12
    assert _close(p["volume"], [12.0])
    # :2713-2725 stress
    stress = [2740384.6153846150, 3317307.6923076920, 5817307.6923076920, -96153.8461538463,
              1346153.8461538465, -192307.6923076927]
    assert _close(p["stress"][0], stress)
    # :2771-2785 body force with gravity (0, 0, -9.81)
    o.phase("body_force", gravity=(0., 0., -9.81))
    body = np.array([-1226.25, -3678.75, -11036.25, -3678.75, -3678.75, -11036.25, -33108.75,
                     -11036.25])
    nodes = o.nodes(8)
    assert _close(nodes[:, 4:6], np.zeros((8, 2))) and _close(nodes[:, 6], body)
    # :2833-2854 internal force with the particle volume reset to 8
    o.set({"volume": np.array([8.0])})
    o.phase("internal_force")
    fint = np.array([[612980.7692307689, 1141826.923076923, 1742788.461538461],
                     [-901442.3076923079, 3521634.615384615, 5420673.076923076],
                     [-2415865.384615385, 612980.7692307703, 12223557.69230769],
                     [1935096.153846153, 108173.0769230771, 3882211.538461538],
                     [2031250, 2079326.923076922, -588942.3076923075],
                     [-2127403.846153846, 6526442.307692306, -1189903.846153845],
                     [-5516826.92307692, -10276442.30769231, -15685096.15384615],
                     [6382211.538461537, -3713942.307692308, -5805288.461538462]])
    nodes = o.nodes(8)
    assert _close(nodes[:, 7:10], fint)
    # :2856-2890 compute_acceleration_velocity, dt = 0.1
    o.phase("node_update", dt=0.1)
    nodes = o.nodes(8)
    v_exp = np.array([[490.3846153846152, 914.4615384615383, 1395.249769230769],
                      [-240.3846153846155, 941.1025641025641, 1448.531820512821],
                      [-214.7435897435898, 57.4871794871796, 1091.557461538462],
                      [516.0256410256410, 32.8461538461539, 1042.275410256410],
                      [541.6666666666666, 559.4871794871794, -148.032282051282],
                      [-189.1025641025641, 586.1282051282051, -94.75023076923067],
                      [-163.4615384615384, -297.4871794871795, -451.7245897435898],
                      [567.3076923076923, -322.1282051282053, -501.0066410256412]])
    a_exp = np.array([[4903.846153846152, 9134.615384615383, 13932.49769230769],
                      [-2403.846153846155, 9391.025641025641, 14445.31820512821],
                      [-2147.435897435898, 544.8717948717959, 10855.57461538462],
                      [5160.256410256409, 288.461538461539, 10342.7541025641],
                      [5416.666666666666, 5544.871794871794, -1580.32282051282],
                      [-1891.025641025641, 5801.282051282051, -1067.502307692307],
                      [-1634.615384615384, -3044.871794871795, -4657.245897435898],
                      [5673.076923076923, -3301.282051282052, -5170.066410256411]])
    assert _close(nodes[:, 10:13], v_exp)
    assert _close(nodes[:, 13:16], a_exp)


def test_chain_catches_a_planted_error():
    """Checks the checker: a 1e-6 error in one nodal force must fail the
    internal-force KAT."""
    o = _one_cell_3d()
    o.phase("initialise")
    nodes = o.nodes(8)
    assert nodes[:, 16].all()
    assert not _close([2031250 * (1 + 1e-6)], [2031250])
