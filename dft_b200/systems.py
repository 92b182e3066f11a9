"""The benchmark systems (synthetic inputs, seeded), shared by bench.py and microbench.

h2_48        H2, Z=1 at +-0.7 bohr on x, 48^3 grid, h = 0.3, centred box, PZ81, multiplicity 1
h2o_128      H2O (O at the origin, O-H 1.81 bohr, HOH 104.5 deg), 128^3 grid, h = 0.2, PBE96,
             multiplicity 1, 5 occupied + 7 extra bands
cluster20    20 nuclei with Z drawn from {1, 6, 7, 8}, positions uniform in a 24-bohr cube centred
             in a 192^3 grid (h = 0.2), minimum separation 2.0 bohr, no nucleus within 1e-12 of a
             node, neutral, multiplicity 1 + (N_e mod 2), PBE96 (seeded numpy generator)
cluster20_clear  the same draw with every nucleus at least 0.08 bohr from the nearest node
cluster20_compact  the same seeded draw in a 14-bohr cube (more vacuum to the box faces)
water        (H2O)_n: n rigid waters, random orientations, O uniform in a 24-bohr cube, O-O >= 5 bohr,
             192^3 grid (h = 0.2), closed shell, PBE96 (seeded numpy generator)
"""
from __future__ import annotations

import math

import numpy as np


def _cube(n, h):
    half = round(0.5 * h * (n - 1), 10)  # e.g. 12.7 for 128 points at h = 0.2
    return (n, n, n), (-half, half) * 3


def h2_48():
    n, b = (48, 48, 48), (-7.05, 7.05) * 3
    return dict(name="h2_48", n=n, bounds=b, Z=[1, 1], xyz=[[-0.7, 0.0, 0.0], [0.7, 0.0, 0.0]], multiplicity=1,
                functional="PZ81", extra_bands=3,
                desc="H2 PZ81 48^3 h=0.3, 1a+1b (multiplicity 1), 4 bands/spin")


def h2o_128(n=128, h=0.2):
    ang = math.radians(104.5 / 2)
    x, z = 1.81 * math.sin(ang), 1.81 * math.cos(ang)
    grid_n, b = _cube(n, h)
    return dict(name=f"h2o_{n}", n=grid_n, bounds=b, Z=[8, 1, 1], xyz=[[0.0, 0.0, 0.0], [x, 0.0, z], [-x, 0.0, z]],
                multiplicity=1, functional="PBE96", extra_bands=7,
                desc=f"H2O PBE96 {n}^3 h={h}, multiplicity 1, 5 occupied + 7 extra bands")


def cluster(natoms=20, n=192, h=0.2, box=24.0, min_sep=2.0, seed=20261203, extra_bands=8, min_node_distance=0.0):
    """min_node_distance > 0 also rejects nuclei closer than that (bohr) to the nearest grid node:
    the point-nucleus potential -Z/r at a node 0.01 bohr from a nucleus is a single-node spike
    (-76 Ha for hydrogen) that binds a spurious grid-scale state."""
    rng = np.random.default_rng(seed)
    grid_n, b = _cube(n, h)
    lo = b[0]
    Z, xyz = [], []
    while len(Z) < natoms:
        p = rng.uniform(-0.5 * box, 0.5 * box, 3)
        if any(np.linalg.norm(p - q) < min_sep for q in xyz):
            continue
        # keep nuclei off grid nodes (the nuclear potential is singular there)
        f = (p - lo) / h
        if np.any(np.abs(f - np.round(f)) * h < 1e-12):
            continue
        if min_node_distance > 0.0 and np.linalg.norm((f - np.round(f)) * h) < min_node_distance:
            continue
        xyz.append(p)
        Z.append(int(rng.choice([1, 6, 7, 8])))
    ne = sum(Z)
    return dict(name=f"cluster{natoms}_{n}", n=grid_n, bounds=b, Z=Z, xyz=[list(map(float, p)) for p in xyz],
                multiplicity=1 + (ne % 2), functional="PBE96", extra_bands=extra_bands,
                desc=f"{natoms}-atom cluster (Z in {{1,6,7,8}}, seed {seed}), {ne} electrons, PBE96 {n}^3 h={h}")


def cluster_clear(**kw):
    """cluster20 with every nucleus at least 0.08 bohr from the nearest grid node."""
    w = cluster(min_node_distance=0.08, **kw)
    w["name"] += "_clear"
    w["desc"] += ", nuclei >= 0.08 bohr from grid nodes"
    return w


def cluster_compact(**kw):
    """The 20-atom draw in a 14-bohr cube instead of 24 (same grid): 12 bohr of vacuum to every
    face instead of 7, which keeps the box-wall states above the Fermi level."""
    kw.setdefault("box", 14.0)
    w = cluster(**kw)
    w["name"] += "_compact"
    w["desc"] += ", nuclei in a 14-bohr cube"
    return w


def water_cluster(nmol=4, n=192, h=0.2, box=24.0, min_sep=5.0, seed=20261204, extra_bands=8):
    """nmol rigid H2O molecules (O-H 1.81 bohr, HOH 104.5 deg), random orientations, O positions
    uniform in a `box`-bohr cube centred in the n^3 grid (h), O-O distances >= min_sep; closed
    shell (multiplicity 1), PBE96.  A bonded, closed-shell cluster: unlike a draw of free atoms,
    its occupied manifold is separated from the empty one by the molecular gap."""
    rng = np.random.default_rng(seed)
    grid_n, b = _cube(n, h)
    lo = b[0]
    ang = math.radians(104.5 / 2)
    local = np.array([[0.0, 0.0, 0.0], [1.81 * math.sin(ang), 0.0, 1.81 * math.cos(ang)],
                      [-1.81 * math.sin(ang), 0.0, 1.81 * math.cos(ang)]])
    Z, xyz, centres = [], [], []
    while len(centres) < nmol:
        c = rng.uniform(-0.5 * box, 0.5 * box, 3)
        if any(np.linalg.norm(c - q) < min_sep for q in centres):
            continue
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))  # random orthogonal frame
        pts = c + local @ q.T
        f = (pts - lo) / h
        if np.any(np.abs(f - np.round(f)) * h < 1e-12):
            continue
        centres.append(c)
        for zz, p in zip((8, 1, 1), pts):
            Z.append(zz)
            xyz.append([float(v) for v in p])
    ne = sum(Z)
    return dict(name=f"water{nmol}_{n}", n=grid_n, bounds=b, Z=Z, xyz=xyz, multiplicity=1, functional="PBE96",
                extra_bands=extra_bands,
                desc=f"(H2O)_{nmol} cluster (random orientations, O in a {box:g}-bohr cube, seed {seed}), "
                     f"{ne} electrons, PBE96 {n}^3 h={h}")


SYSTEMS = {"h2_48": h2_48, "h2o_128": h2o_128, "cluster20": cluster, "cluster20_clear": cluster_clear,
           "cluster20_compact": cluster_compact, "water": water_cluster}


def get(name, **kw):
    return SYSTEMS[name](**kw)
