"""GPU: the learned Poisson start.

* The network's forward pass and parameter gradient against the CPU oracle
  (oracle/pnet_reference.py, PyTorch FP32 with the same BF16 roundings), at BF16 tolerance.
* The coarse-grid start: Jacobi from it stops with the unchanged rule in fewer sweeps and
  lands as close to the converged potential as the cold start does.
* Training on the device lowers the validation loss below the coarse start's, and the
  trained network's start saves Jacobi sweeps over the coarse start alone.
* The SCF with each start converges to the cold-start energy.
"""
import numpy as np
import pytest

import dft_b200
from oracle import pnet_reference as R

pytestmark = pytest.mark.gpu


def _random_params(seed):
    rng = np.random.default_rng(seed)
    offs, total = R.offsets()
    p = np.zeros(total, dtype=np.float32)
    for (typ, cin, cout), (wo, bo) in zip(R.LAYERS, offs):
        fan = R.TAPS[typ] * cin
        n = R.TAPS[typ] * cin * cout
        p[wo:wo + n] = rng.uniform(-1, 1, n) * np.sqrt(3.0 / fan)
        p[bo:bo + cout] = rng.uniform(-0.1, 0.1, cout)
    return p


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_param_count_matches_oracle(engine):
    net = dft_b200.PoissonNet(engine)
    assert net.num_params == R.offsets()[1]
    p = net.get_params()
    net.set_params(p * 2)
    assert np.array_equal(net.get_params(), p * 2)


@pytest.mark.parametrize("tensor_cores", [1, 0], ids=["tcgen05", "cuda_cores"])
@pytest.mark.parametrize("shape", [(10, 9, 7), (37, 34, 21)])
def test_forward_and_gradient_vs_oracle(engine, shape, tensor_cores):
    engine.set_tuning("network_tensor_cores", tensor_cores)
    net = dft_b200.PoissonNet(engine)
    p = _random_params(11)
    net.set_params(p)
    N = int(np.prod(shape))
    rng = np.random.default_rng(12)
    x = rng.uniform(-1, 1, (N, 2)).astype(np.float32)
    t = (0.1 * rng.standard_normal(N)).astype(np.float32)
    loss, grad, y = net.loss_grad(shape, x, t)
    l_ref, g_ref, y_ref = R.loss_grad(p, x, t, shape)
    assert _rel(y, y_ref) < 1e-2
    assert abs(loss - l_ref) < 1e-2 * l_ref
    offs, _ = R.offsets()
    for (typ, cin, cout), (wo, bo) in zip(R.LAYERS, offs):
        n = R.TAPS[typ] * cin * cout
        assert _rel(grad[wo:wo + n], g_ref[wo:wo + n]) < 3e-2, (typ, cin, cout)
        assert _rel(grad[bo:bo + cout], g_ref[bo:bo + cout]) < 3e-2, (typ, cin, cout, "bias")
    engine.set_tuning("network_tensor_cores", 1)


def _h2_grid(n=48, half=7.05):
    return dft_b200.CartesianGrid(n, n, n, -half, half, -half, half, -half, half)


def test_coarse_start_saves_sweeps(engine):
    g = _h2_grid()
    N = g.getSize()
    rho = engine.array(N)
    engine.synthetic_density(g, 7, rho)
    vstar = engine.array(N)
    engine.hartree(g, rho, vstar, 1e-13, 200000)
    ref = vstar.to_host()
    vc = engine.array(N)
    sw_cold, _ = engine.hartree(g, rho, vc)
    vg = engine.array(N)
    engine.poisson_start(g, None, rho, vg)
    start = vg.to_host()
    # sharp peaks (widths down to one fine spacing) are not resolved on the coarse levels;
    # the start is judged by the sweeps it saves and where Jacobi ends from it
    assert np.linalg.norm(start - ref) < 0.1 * np.linalg.norm(ref)
    sw_guess, _ = engine.hartree_from_guess(g, rho, vg)
    print(f"cold {sw_cold} sweeps, coarse start {sw_guess} sweeps")
    assert sw_guess < 0.8 * sw_cold
    err_cold = np.max(np.abs(vc.to_host() - ref))
    err_guess = np.max(np.abs(vg.to_host() - ref))
    assert err_guess <= 2.0 * err_cold + 1e-9


@pytest.mark.parametrize("n,half", [(48, 7.05), (64, 6.3), (33, 4.0)])
def test_multigrid_start(engine, n, half):
    """V-cycles bring the start to the Jacobi stop rule: a few fine sweeps remain, and the
    result is at least as close to the converged potential as the cold-start Jacobi result."""
    g = _h2_grid(n, half)
    N = g.getSize()
    rho = engine.array(N)
    engine.synthetic_density(g, 17, rho)
    vstar = engine.array(N)
    engine.hartree(g, rho, vstar, 1e-13, 400000)
    ref = vstar.to_host()
    vc = engine.array(N)
    sw_cold, _ = engine.hartree(g, rho, vc)
    vm = engine.array(N)
    info = engine.poisson_start(g, None, rho, vm, multigrid_cycles=40)
    sw_mg, _ = engine.hartree_from_guess(g, rho, vm)
    err_cold = np.max(np.abs(vc.to_host() - ref))
    err_mg = np.max(np.abs(vm.to_host() - ref))
    print(f"n={n}: cold {sw_cold} sweeps (err {err_cold:.2e}); multigrid {info} then {sw_mg} sweeps (err {err_mg:.2e})")
    assert info["multigrid_cycles"] < 40 and info["residual"] < 0.5e-8
    assert sw_mg <= 5
    assert err_mg <= err_cold + 1e-9


def test_training_beats_coarse_start(engine):
    """The network trained on the device lowers the validation error of the start, and the
    multigrid cycles that follow start from a smaller residual."""
    g = _h2_grid()
    net = dft_b200.PoissonNet(engine, seed=3)
    rep = net.train([g], samples=48, validation=8, epochs=12, batch=4, lr=3e-3, lr_min=1e-4, seed=99,
                    smooth_sweeps=0, mse_weight=1.0)
    assert rep["steps"] == 12 * 10
    assert rep["val_loss"] < 0.5 * rep["val_loss_coarse"], rep
    N = g.getSize()
    rho, v = engine.array(N), engine.array(N)
    res_c = res_n = 0.0
    cyc_c = cyc_n = 0
    for seed in (1001, 1002, 1003):
        engine.synthetic_density(g, seed, rho)
        res_c += engine.poisson_start(g, None, rho, v, multigrid_cycles=2)["residual"]
        res_n += engine.poisson_start(g, net, rho, v, multigrid_cycles=2)["residual"]
        cyc_c += engine.poisson_start(g, None, rho, v, multigrid_cycles=40)["multigrid_cycles"]
        cyc_n += engine.poisson_start(g, net, rho, v, multigrid_cycles=40)["multigrid_cycles"]
    print(rep, f"residual after 2 cycles: coarse {res_c:.3e} network {res_n:.3e}; cycles to tolerance: "
               f"coarse {cyc_c} network {cyc_n}")
    assert res_n < res_c
    assert cyc_n <= cyc_c


def test_scf_with_each_poisson_start(engine):
    g = dft_b200.CartesianGrid(32, 32, 32, -6.2, 6.2, -6.2, 6.2, -6.2, 6.2)
    m = dft_b200.Molecule()
    m.addNucleus(1, -0.7, 0.0, 0.0)
    m.addNucleus(1, 0.7, 0.0, 0.0)
    energies, sweeps = {}, {}
    for mode in (dft_b200.POISSON_COLD, dft_b200.POISSON_PREVIOUS, dft_b200.POISSON_COARSE,
                 dft_b200.POISSON_HYBRID, dft_b200.POISSON_MULTIGRID):
        o = dft_b200.default_scf_options(stop_abs_de=1e-6, poisson_start=mode)
        r = engine.scf_molecule(g, m, 0, 1, "PZ81", o)
        energies[mode] = r.total
        sweeps[mode] = sum(h["poisson_sweeps_in"] + h["poisson_sweeps_out"] for h in r.history)
    print(energies, sweeps)
    for mode, e in energies.items():
        assert abs(e - energies[dft_b200.POISSON_COLD]) < 2e-5, (mode, energies)
    assert sweeps[dft_b200.POISSON_HYBRID] < 0.6 * sweeps[dft_b200.POISSON_COLD], sweeps
    assert sweeps[dft_b200.POISSON_MULTIGRID] < 0.01 * sweeps[dft_b200.POISSON_COLD], sweeps


@pytest.mark.parametrize("case", ["h2_closed", "h3_doublet"])
def test_pulay_mixer_same_energy(engine, case):
    """The Pulay mixer and the adaptive eigensolver tolerance reach the linear mixer's energy."""
    g = dft_b200.CartesianGrid(28, 28, 28, -5.4, 5.4, -5.4, 5.4, -5.4, 5.4)
    m = dft_b200.Molecule()
    if case == "h2_closed":
        m.addNucleus(1, -0.7, 0.0, 0.0)
        m.addNucleus(1, 0.7, 0.0, 0.0)
        mult = 1
    else:
        m.addNucleus(1, -1.6, 0.0, 0.0)
        m.addNucleus(1, 0.0, 0.1, 0.0)
        m.addNucleus(1, 1.6, 0.0, 0.0)
        mult = 2
    res = {}
    for mixer, adaptive in ((0, 0), (1, 0), (1, 1)):
        o = dft_b200.default_scf_options(stop_abs_de=1e-8, poisson_start=dft_b200.POISSON_MULTIGRID, mixer=mixer,
                                         adaptive_eig_tol=adaptive)
        r = engine.scf_molecule(g, m, 0, mult, "PBE96", o)
        res[(mixer, adaptive)] = (r.total, r.iterations)
    print(case, res)
    e0 = res[(0, 0)][0]
    for k, (e, it) in res.items():
        assert abs(e - e0) < 1e-6, (k, res)
    assert res[(1, 0)][1] <= res[(0, 0)][1]


def test_fermi_smearing_limits(engine):
    """A small smearing temperature reproduces the integer-occupation energy of a gapped
    molecule; a larger one still converges."""
    g = dft_b200.CartesianGrid(28, 28, 28, -5.4, 5.4, -5.4, 5.4, -5.4, 5.4)
    m = dft_b200.Molecule()
    m.addNucleus(1, -0.7, 0.0, 0.0)
    m.addNucleus(1, 0.7, 0.0, 0.0)
    e = {}
    for kt in (0.0, 1e-4, 2e-2):
        o = dft_b200.default_scf_options(stop_abs_de=1e-8, poisson_start=dft_b200.POISSON_MULTIGRID, mixer=1,
                                         smearing_kt=kt)
        r = engine.scf_molecule(g, m, 0, 1, "PZ81", o)
        e[kt] = (r.total, r.iterations)
    print(e)
    assert abs(e[1e-4][0] - e[0.0][0]) < 1e-6
    assert np.isfinite(e[2e-2][0]) and e[2e-2][1] < 100


def test_multigrid_graph_replay_identical(engine):
    """Replaying the captured multigrid cycle gives the same potential, bit for bit, as
    launching its kernels one by one."""
    n = (40, 36, 44)
    g = dft_b200.CartesianGrid(*n, -5.85, 5.85, -5.25, 5.25, -6.45, 6.45)
    N = g.getSize()
    rho = engine.array(N)
    engine.synthetic_density(g, 11, rho)
    out = {}
    try:
        for graphs in (0, 1, 1):  # the second graph run replays the cached capture
            engine.set_tuning("multigrid_graphs", graphs)
            v = engine.array(N)
            info = engine.poisson_start(g, None, rho, v, multigrid_cycles=6)
            out.setdefault(graphs, []).append((v.to_host(), info["multigrid_cycles"]))
    finally:
        engine.set_tuning("multigrid_graphs", 1)
    ref, cyc = out[0][0]
    for v, c in out[1]:
        assert c == cyc and np.array_equal(v, ref)
