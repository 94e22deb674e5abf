"""The closure MLP on the tensor cores (tcgen05) against its FP64 oracle.

The oracle's gradients are pinned by central finite differences (CPU test); the GPU kernels
are compared with the oracle that rounds to BF16 where the kernels hold BF16 values.
Tolerance: 2e-2 relative (Frobenius norm per parameter block) for gradients, 1e-2 for
outputs; the differences come from FP32 accumulation order, from the special-function unit's
tanh (tanh.approx.f32, absolute error about 2^-11) inside GELU, and from activations that land
on the other side of a BF16 rounding boundary.
"""
import numpy as np
import pytest

from oracle import closure_oracle as co


def _data(n, seed):
    rng = np.random.default_rng(seed)
    X = co.bf16(rng.standard_normal((n, co.NIN)))
    T = np.stack([np.sin(X[:, 0]) + 0.3 * X[:, 1] * X[:, 2], np.cos(X[:, 3]) - 0.2 * X[:, 4]], axis=1)
    return X, T


def test_oracle_gradients_finite_differences():
    X, T = _data(37, 1)
    p = co.init_params(3)
    g, _ = co.gradients(p, X, T, rounding=False)
    rng = np.random.default_rng(0)
    for idx in rng.choice(co.NPARAM, 40, replace=False):
        e = np.zeros(co.NPARAM)
        e[idx] = 1e-6
        fd = (co.loss(p + e, X, T, rounding=False) - co.loss(p - e, X, T, rounding=False)) / 2e-6
        assert abs(fd - g[idx]) <= 1e-6 + 1e-5 * abs(fd)


def test_gelu_tanh_form_against_erf_form():
    """The network's GELU is the tanh form of Hendrycks and Gimpel (2016); it stays within
    4.8e-4 of the erf form everywhere, and its derivative matches finite differences."""
    x = np.linspace(-12, 12, 480001)
    assert np.abs(co.gelu(x) - co.gelu_erf(x)).max() <= 4.8e-4
    h = 1e-6
    fd = (co.gelu(x + h) - co.gelu(x - h)) / (2 * h)
    assert np.abs(fd - co.gelu_grad(x)).max() <= 1e-8


def _blocks(v):
    out, k = {}, 0
    for name, shape in co.SHAPES:
        n = int(np.prod(shape))
        out[name] = v[k:k + n]
        k += n
    return out


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 100, 128, 1000, 70000])
def test_forward_and_gradients_match_oracle(require_gpu, n):
    import torch
    import dmplex_b200.closure as cl
    X, T = _data(n, n)
    p = co.init_params(7)
    p[co.NH * co.NIN:co.NH * co.NIN + co.NH] = 0.1  # nonzero b1
    mlp = cl.ClosureMLP(p.astype(np.float32))
    assert mlp.info()["forward_ctas_per_sm"] >= 6  # the persistent grid fills the SMs
    Xd = torch.from_numpy(X.astype(np.float32)).to(torch.bfloat16).cuda().contiguous()
    Td = torch.from_numpy(T.astype(np.float32)).cuda().contiguous()
    pf = mlp.params().astype(np.float64)
    Y = mlp.forward(Xd).cpu().numpy()
    Yo, _ = co.forward(pf, X)
    assert _rel(Y, Yo) <= 1e-2
    g, loss = mlp.gradients(Xd, Td)
    go, lo = co.gradients(pf, X, T)
    assert abs(loss - lo) <= 1e-2 * lo
    gb, gob = _blocks(g), _blocks(go)
    for name, _ in co.SHAPES:
        assert _rel(gb[name], gob[name]) <= 2e-2, name


@pytest.mark.gpu
def test_training_reduces_loss(require_gpu):
    import torch
    import dmplex_b200.closure as cl
    X, T = _data(65536, 5)
    mlp = cl.ClosureMLP(seed=1)
    Xd = torch.from_numpy(X.astype(np.float32)).to(torch.bfloat16).cuda().contiguous()
    Td = torch.from_numpy(T.astype(np.float32)).cuda().contiguous()
    first = mlp.train_step(Xd, Td, 3e-3)
    for _ in range(300):
        last = mlp.train_step(Xd, Td, 3e-3)
    assert np.isfinite(last) and last < 0.1 * first


@pytest.mark.gpu
@pytest.mark.parametrize("state_bits", [64, 32])
def test_ensemble_features_match_oracle(require_gpu, state_bits):
    """The closure's 24 inputs from an ensemble's member states against the same quantities
    built from the CPU oracle's work vectors (K via B - g h, q at the vertices), rounded to
    BF16 like the kernel; exact."""
    import torch
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    from dmplex_b200.coarsen import edge_geometry
    from oracle.oracle import Oracle
    from conftest import tables, trisk_grid
    si = w.si_parameters()
    g = trisk_grid(3, True)
    t = tables(3, "trisk", "cell", True, None, **si)
    m = d.TRiSKShallowWater(g, pv_flux="trisk", kinetic_energy="cell", **si)
    o = Oracle(t)
    states = w.ensemble_members(g, 2, 3, degree=6)
    if state_bits == 32:  # the ensemble stores float: the oracle sees the rounded states
        states = [y.astype(np.float32).astype(np.float64) for y in states]
    ens = d.Ensemble([(m, 2, 100.0, 1)], state_bits=state_bits)
    for k, y in enumerate(states):
        ens.set_member(0, k, y)
    geom = edge_geometry(g)
    norm = np.concatenate([np.zeros(24), np.ones(24), [1.0, 1.0]])
    X = torch.empty((g.ne * 2, 24), dtype=torch.bfloat16, device="cuda")
    ens.features(0, X, norm, geom)
    got = X.float().cpu().numpy().astype(np.float64).reshape(g.ne, 2, 24)
    ne = g.ne
    te, tw = t["trisk_edges"] - 1, t["trisk"]
    ec, ev = t["edge_cells"] - 1, t["edge_vertices"] - 1
    for k, y in enumerate(states):
        o.tendency(y)
        wk = o.work()
        if state_bits == 32:  # the ensemble stores its work vectors as float too
            wk = {key: v.astype(np.float32).astype(np.float64) for key, v in wk.items()}
        u, h = y[:ne], y[ne:]
        h0, h1 = h[ec[:, 0]], h[ec[:, 1]]
        q0, q1 = wk["qv"][ev[:, 0]], wk["qv"][ev[:, 1]]
        K0, K1 = wk["B"][ec[:, 0]] - t["gravity"] * h0, wk["B"][ec[:, 1]] - t["gravity"] * h1
        f = np.zeros((ne, 24))
        f[:, 0] = u
        f[:, 1:11] = np.where(tw != 0, u[te] - u[:, None], 0.0)
        f[:, 11], f[:, 12] = (h0 + h1) / 2, h1 - h0
        f[:, 13], f[:, 14] = (q0 + q1) / 2, q1 - q0
        f[:, 15], f[:, 16] = (K0 + K1) / 2, K1 - K0
        f[:, 17:] = geom
        assert np.array_equal(got[:, k, :], co.bf16(f))


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_the_closure_stays_usable(require_gpu):
    """A tensor-core wait that runs out (here: the first operation of tile 3 is not issued, so
    nothing arrives on its barrier) ends the call with TRISK_ERR_TIMEOUT after half a second,
    without a trap; the CTA frees its tensor memory, and the next call on the same closure
    returns the same rows as before and matches the oracle."""
    import torch
    import dmplex_b200 as d
    import dmplex_b200.closure as cl
    X, _ = _data(1000, 9)
    mlp = cl.ClosureMLP(co.init_params(4).astype(np.float32))
    Xd = torch.from_numpy(X.astype(np.float32)).to(torch.bfloat16).cuda().contiguous()
    before = mlp.forward(Xd).clone()
    mlp.expire_wait_once(3)
    with pytest.raises(d.TriskError) as err:
        mlp.forward(Xd)
    assert err.value.status == 5
    after = mlp.forward(Xd)
    assert torch.equal(before, after)
    Yo, _ = co.forward(mlp.params().astype(np.float64), X)
    assert _rel(after.cpu().numpy(), Yo) <= 1e-2


@pytest.mark.gpu
def test_forward_large_batch_rows_are_independent(require_gpu):
    """4,194,304 rows (201 MB of features, more than the L2) through the persistent inference
    grid: every row equals the same row computed in a small batch, bit for bit (each row is one
    thread's, whatever tile and CTA it falls in), and a sample matches the oracle."""
    import torch
    import dmplex_b200.closure as cl
    n = 4_194_304
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    Xd = torch.randn((n, co.NIN), device="cuda", generator=g).to(torch.bfloat16).contiguous()
    mlp = cl.ClosureMLP(co.init_params(2).astype(np.float32))
    Y = mlp.forward(Xd)
    for start in (0, 1_000_003, n - 777):
        part = mlp.forward(Xd[start:start + 777].contiguous())
        assert torch.equal(part, Y[start:start + 777])
    idx = torch.arange(0, n, 4099, device="cuda")
    Xs = Xd[idx].float().cpu().numpy().astype(np.float64)
    Yo, _ = co.forward(mlp.params().astype(np.float64), Xs)
    assert _rel(Y[idx].cpu().numpy(), Yo) <= 1e-2
