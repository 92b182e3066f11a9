"""CPU: the synthetic workloads and the bench's Poisson oracle tolerance."""
import math

import numpy as np

from dft_b200 import systems


def test_h2_48_spacing_is_exact():
    w = systems.get("h2_48")
    (n, _, _), b = w["n"], w["bounds"]
    assert abs((b[1] - b[0]) / (n - 1) - 0.3) < 1e-15


def test_cluster_draws_respect_their_rules():
    for name, min_node in (("cluster20", 0.0), ("cluster20_clear", 0.08)):
        w = systems.get(name)
        xyz = np.array(w["xyz"])
        assert len(w["Z"]) == 20 and set(w["Z"]) <= {1, 6, 7, 8}
        d = np.linalg.norm(xyz[:, None, :] - xyz[None, :, :], axis=-1) + 1e9 * np.eye(20)
        assert d.min() >= 2.0
        assert np.all(np.abs(xyz) <= 12.0)
        assert w["multiplicity"] == 1 + sum(w["Z"]) % 2
        h = (w["bounds"][1] - w["bounds"][0]) / (w["n"][0] - 1)
        f = (xyz - w["bounds"][0]) / h
        assert np.all(np.linalg.norm((f - np.round(f)) * h, axis=1) >= min_node)
    assert systems.get("cluster20")["Z"] == systems.cluster()["Z"]  # the seeded draw is stable


def test_tight_poisson_tolerance():
    import bench
    w = systems.get("h2_48")
    rho = math.cos(math.pi / 47)
    assert abs(bench.jacobi_tight_tol(w) - 1e-8 * (1 - rho)) < 1e-20
