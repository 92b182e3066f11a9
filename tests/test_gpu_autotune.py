"""GPU: the launch-shape autotuner (dft_autotune).  Every variant it times gives bit-identical
results, so the choice changes speed only: the SCF energy with the autotuner on is the same
number as with it off, the choice is the fastest variant it timed, and a second call for the
same grid is remembered."""
import numpy as np
import pytest

import dft_b200

pytestmark = pytest.mark.gpu


def test_autotune_picks_fastest_and_remembers(engine):
    g = dft_b200.CartesianGrid(40, 36, 34, -6.0, 6.0, -5.4, 5.4, -5.0, 5.0)
    r = engine.autotune(g, 6)
    print(r)
    assert not r["cached"]
    times = [v for v in list(r["hpsi_ms"]) + list(r["hpsi_tma_ms"]) + [r["hpsi_prefetch_ms"]]
             + list(r["hpsi_zchunk_ms"]) if v >= 0]
    if r["hpsi_zchunk"] > 0:
        chosen = r["hpsi_zchunk_ms"][[16, 32, 64, 96, 192].index(r["hpsi_zchunk"])]
    elif r["hpsi_variant"] == 3:
        chosen = r["hpsi_prefetch_ms"]
    elif r["hpsi_variant"] == 2:
        chosen = r["hpsi_tma_ms"][[1, 2, 4, 8].index(r["hpsi_bands_per_thread"])]
    else:
        chosen = r["hpsi_ms"][[1, 2, 4].index(r["hpsi_bands_per_thread"])]
    assert chosen == min(times)
    assert all(v >= 0 for v in r["hpsi_tma_ms"][:3])  # nx = 40 is even: the TMA ring applies
    spl = dict(zip([-2, -1, 1, 2, 4, 8], r["jacobi_us_per_sweep"]))
    assert spl[r["jacobi_sweeps_per_launch"]] == min(v for v in spl.values() if v >= 0)
    assert engine.autotune(g, 6)["cached"]


def test_scf_energy_unchanged_by_autotune(engine):
    g = dft_b200.CartesianGrid(30, 30, 30, -5.8, 5.8, -5.8, 5.8, -5.8, 5.8)
    m = dft_b200.Molecule()
    m.addNucleus(1, -0.7, 0.011, 0.0)
    m.addNucleus(1, 0.7, 0.011, 0.0)
    e = []
    for at in (0, 1):
        r = engine.scf_molecule(g, m, 0, 1, "PZ81", dft_b200.default_scf_options(stop_abs_de=1e-7, autotune=at))
        e.append((r.total, r.eigenvalues))
    assert e[0][0] == e[1][0] and np.array_equal(e[0][1], e[1][1])
