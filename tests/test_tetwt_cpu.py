"""CPU checks of the tetrahedron-weight oracle: the Rath-Freeman histogram of
one tetrahedron against Monte Carlo sampling, and the volume sum rule."""
import numpy as np

from ecalj_b200 import synth
from oracle import tetwt as tw


def test_histogram_matches_monte_carlo():
    rng = np.random.default_rng(1)
    checked = 0
    for _ in range(8):
        kv = rng.normal(size=(4, 3))
        ea, eb = rng.uniform(-1.0, 0.4, 4), rng.uniform(-0.3, 1.5, 4)
        x = 0.5 * (ea - eb)
        fr = np.linspace(-0.2, 1.2, 29)
        wt = tw.lindtet6(kv, ea, eb, x, 0.0, 0.0, fr)
        n = 200000
        u = rng.dirichlet([1, 1, 1, 1], n)
        vol = abs(np.linalg.det(np.stack([kv[i] - kv[3] for i in range(3)], 1))) / 6
        inside = ((u @ ea) < 0) & ((u @ eb) > 0)
        h, _ = np.histogram(-(u[inside] @ x), bins=fr)
        mc = h / n * vol
        sig = np.sqrt(np.maximum(h, 1)) / n * vol                    # Poisson error of each bin
        assert np.all(np.abs(wt - mc) <= 5 * sig + 1e-12)
        assert abs(wt.sum() - inside.mean() * vol) <= 5 * np.sqrt(inside.mean() / n) * vol + 1e-12
        checked += 1
    assert checked == 8


def test_fully_inside_tetrahedron_gives_its_volume():
    kv = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    ea = np.array([-0.5, -0.4, -0.3, -0.2])
    eb = np.array([0.3, 0.5, 0.4, 0.6])
    wt = tw.lindtet6(kv, ea, eb, 0.5 * (ea - eb), 0.0, 0.0, np.linspace(0.0, 1.0, 11))
    assert abs(wt.sum() - 1.0 / 6.0) <= 1e-12


def test_mesh_generator():
    idt, q, ek, ekq = synth.tetra_mesh(2)
    assert idt.shape == (48, 4) and q.shape == (27, 3) and ek.shape == ekq.shape == (27, 6)
    vols = [abs(np.linalg.det(np.stack([q[t[i]] - q[t[3]] for i in range(3)], 1))) / 6 for t in idt]
    assert abs(sum(vols) - 1.0) <= 1e-12 and min(vols) > 0
