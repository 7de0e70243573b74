"""GPU tests of the property engine: table splines (THERM_PROP_UPDATE)
against the FP64 oracle, the MLP training kernels' loss and gradient against
the FP64 numpy reference, training convergence, the tcgen05 tensor-core
inference (BF16 hi/lo operands, FP32 accumulation) against the FP64 forward
of the same parameters, the per-bin error gate at its 1e-4 bound, and the
out-of-table error path."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def table():
    from chapsim1ww_b200.props import synthetic_table
    return synthetic_table(4096)


@pytest.fixture(scope="module")
def engine(table):
    _need_gpu()
    from chapsim1ww_b200 import PropertyEngine
    return PropertyEngine(*table)


def _oracle_update(table, h):
    from oracle import pyoracle
    L = pyoracle.load()
    P = ctypes.c_void_p
    L.oracle_therm_prop_update.argtypes = [ctypes.c_int] + [P] * 5 + [ctypes.c_int64] + [P] * 5
    L.oracle_therm_prop_update.restype = ctypes.c_int64
    H, T, D, M, K, _ = [np.ascontiguousarray(c) for c in table]
    out = [np.full(len(h), -7.0) for _ in range(4)]
    bad = L.oracle_therm_prop_update(len(H), H.ctypes.data, T.ctypes.data, D.ctypes.data, M.ctypes.data,
                                     K.ctypes.data, len(h), h.ctypes.data, *[o.ctypes.data for o in out])
    return bad, out


def test_table_update_matches_oracle(engine, table):
    import torch
    rng = np.random.default_rng(3)
    h = rng.uniform(-0.9999, 0.9999, 200_000)
    h[:7] = [0.0, 3e-11, -5e-11, 0.1, -0.1, 0.5, H1 := table[0][1] * 0.5 + table[0][2] * 0.5]
    bad_o, (To, Do, Mo, Ko) = _oracle_update(table, h)
    assert bad_o == 0
    dev = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")
    hd = dev(h)
    T, rho, mu, k = (dev(np.full(len(h), -7.0)) for _ in range(4))
    engine.update(hd, T, rho, mu, k)
    for g, o in ((T, To), (rho, Do), (mu, Mo), (k, Ko)):
        g = g.cpu().numpy()
        assert np.abs(g - o).max() <= 1e-13 * np.abs(o).max()
    assert T[0].item() == -7.0 and T[1].item() == -7.0  # |h| < 1e-10 left unchanged


def test_out_of_table_is_an_error(engine):
    import torch
    from chapsim1ww_b200 import ChapsimError
    h = torch.tensor([0.2, 1.2, -3.0, 1.0], dtype=torch.float64, device="cuda")
    outs = [torch.full((4,), -7.0, dtype=torch.float64, device="cuda") for _ in range(4)]
    with pytest.raises(ChapsimError) as e:
        engine.update(h, *outs)
    assert "RANGE" in str(e.value)
    assert engine.update(h, *outs, raise_on_range=False) == 3
    assert outs[0][1].item() == -7.0 and outs[0][0].item() != -7.0


def test_loss_and_gradient_match_fp64_reference(engine):
    from oracle import mlp_ref
    rng = np.random.default_rng(7)
    p = rng.normal(0, 0.3, mlp_ref.NPARAM).astype(np.float32)
    norm = np.array([0.0, 1.0] + [0.0] * 5 + [1.0] * 5 + [0.0] * 30)
    engine.set_params(p, norm)
    x = rng.uniform(-1, 1, 300).astype(np.float32)
    t = rng.normal(0, 1, (300, 5)).astype(np.float32)
    loss, g = engine.loss_grad(x, t)
    lr, gr = mlp_ref.loss_and_grad(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - lr) <= 1e-5 * lr
    assert np.linalg.norm(g - gr) <= 2e-4 * np.linalg.norm(gr)
    assert np.abs(g - gr).max() <= 1e-3 * np.abs(gr).max()


def test_tensor_core_inference_matches_fp64_forward(engine):
    """Random parameters and base: the tcgen05 kernel (every bin on the
    model) against the FP64 forward.  A layout or descriptor error gives O(1)
    differences; the split operands and tanh.approx.f32 leave about 1e-5."""
    import torch
    from oracle import mlp_ref
    rng = np.random.default_rng(17)
    p = rng.normal(0, 0.3, mlp_ref.NPARAM).astype(np.float32)
    base = rng.normal(0, 0.5, (5, 6))
    norm = np.concatenate([[0.0, 1.0], rng.normal(0, 0.2, 5), np.full(5, 0.05), base.ravel()])
    engine.set_params(p, norm)
    nb, _ = engine.gate(tol=1e9, nbins=64)
    assert nb == 64
    h = rng.uniform(-0.999, 0.999, 5000)  # a partial last tile (5000 = 39 x 128 + 8)
    hd = torch.tensor(h, dtype=torch.float64, device="cuda")
    outs = [torch.zeros(len(h), dtype=torch.float64, device="cuda") for _ in range(5)]
    engine.update(hd, *outs[:4], cp=outs[4], mode=1)
    ref = mlp_ref.properties(p.astype(np.float64), norm, h)
    for o in range(5):
        got = outs[o].cpu().numpy()
        err = np.abs(got - ref[:, o]).max() / np.abs(ref[:, o]).max()
        assert err <= 1e-4, (o, err)


def test_training_gate_and_fallback(engine, table):
    """Training on 65,536 table samples (seed 2) reaches the 1e-4 bound (error
    relative to each output's largest magnitude over the table) in at least
    200 of 256 h-bins for T, rho, mu and k, the outputs THERM_PROP_UPDATE
    produces; at random points the gated update stays within 2e-4 of the
    table (the gate samples 128 points per bin)."""
    import torch
    loss = engine.train(nsamples=65536, seed=2, steps=20000, lr=3e-3)
    nb, worst = engine.gate(tol=1e-4, nbins=256)
    bins, errs = engine.gate_outputs()
    print(f"trained: loss {loss:.3e}, bins passing (T, rho, mu, k) {nb}/256, per output {bins}, "
          f"worst per output {['%.2e' % e for e in errs]}")
    assert nb >= 200, (nb, bins, errs)
    rng = np.random.default_rng(11)
    h = rng.uniform(-0.999, 0.999, 100_000)
    hd = torch.tensor(h, dtype=torch.float64, device="cuda")
    got = [torch.zeros(len(h), dtype=torch.float64, device="cuda") for _ in range(4)]
    tab = [torch.zeros(len(h), dtype=torch.float64, device="cuda") for _ in range(4)]
    engine.update(hd, *got, mode=1)
    engine.update(hd, *tab)
    for o in range(4):
        a, b = got[o].cpu().numpy(), tab[o].cpu().numpy()
        assert np.abs(a - b).max() <= 2e-4 * np.abs(b).max(), o
    # gate with a zero bound: every bin falls back to the table splines, bitwise
    nb, _ = engine.gate(tol=0.0, nbins=64)
    assert nb == 0
    engine.update(hd, *got, mode=1)
    for a, b in zip(got, tab):
        assert torch.equal(a, b)


def test_network_gain_over_polynomial_base(table):
    """What the trained network gains over the model without it: the same
    normalisation and degree-5 polynomial base with the network's output
    layer zeroed (a residual of zero) against the trained network, both
    evaluated on the tensor cores and gated at 1e-4 against the table.  The
    network lowers the worst error of T, rho, mu and k by more than 10x and
    clears more h-bins."""
    _need_gpu()
    from chapsim1ww_b200 import PropertyEngine
    from oracle import mlp_ref
    e = PropertyEngine(*table)
    e.train(nsamples=65536, seed=2, steps=20000, lr=3e-3)
    nb_net, _ = e.gate(tol=1e-4, nbins=256)
    bins_net, errs_net = e.gate_outputs()
    p, norm = e.get_params()
    o_w3 = mlp_ref.NH + mlp_ref.NH + mlp_ref.NH * mlp_ref.NH + mlp_ref.NH
    p0 = p.copy()
    p0[o_w3:] = 0.0  # W3 and b3: the network adds nothing to the base
    e.set_params(p0, norm)
    nb_base, _ = e.gate(tol=1e-4, nbins=256)
    bins_base, errs_base = e.gate_outputs()
    print(f"bins cleared for T, rho, mu, k: base alone {nb_base}/256, with the network {nb_net}/256; "
          f"worst error per output (T, rho, mu, k, cp) base {['%.2e' % x for x in errs_base]}, "
          f"network {['%.2e' % x for x in errs_net]}")
    assert nb_net > nb_base and nb_net >= 200
    for o in range(4):
        assert errs_net[o] * 10 <= errs_base[o], (o, errs_net[o], errs_base[o])
    e.close()
