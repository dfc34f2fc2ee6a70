"""Differentiable form: nkg_graph_set_weights, nkg_pagerank_run_ex and the
adjoint nkg_pagerank_adjoint, against the oracle's FP64 host adjoint and
central finite differences of the forward.

Bars: FP64 and FP32_REFINE gradients within 1e-9 of the largest oracle
gradient (max abs), FP32 within 1e-4; finite differences within
1e-7 + 1e-5 |fd| (oracle forward, h = 1e-5) or 1e-5 relative to the largest
checked gradient (GPU FP64 forward, h = 1e-4)."""
import numpy as np
import pytest

from networkit_b200 import _capi, generators

pytestmark = pytest.mark.gpu

DAMP = 0.85


def weighted_rmat(scale, ef, seed):
    return generators.with_uniform_weights(generators.rmat_directed(scale, ef, seed=seed),
                                           seed=seed + 1)


def sum_x(csr, p, teleport, distribute):
    """sum(x) of the forward fixed point from its normalised scores."""
    sp = float(p[csr.outdeg == 0].sum())
    tau = 1.0 if teleport is None else float(teleport.sum())
    return (1 - DAMP) * tau / (1 - DAMP + DAMP * sp * (1 - (tau if distribute else 0.0)))


def random_teleport(z, seed):
    t = np.random.default_rng(seed).random(z) + 0.05
    return t / t.sum()


def oracle_grads(oracle_mod, csr, g, distribute, teleport):
    o = oracle_mod.pagerank(csr, tol=1e-14, norm=0, distribute_sinks=distribute,
                            teleport=teleport, max_iterations=5000)
    p = o.scores
    x = p * sum_x(csr, p, teleport, distribute)
    _, gw, gt, _ = oracle_mod.adjoint(csr, x, g, damp=DAMP, distribute_sinks=distribute,
                                      teleport=teleport, tol=1e-15)
    return p, gw, gt


PRECS = {"fp64": _capi.NKG_PREC_FP64, "refine": _capi.NKG_PREC_FP32_REFINE,
         "fp32": _capi.NKG_PREC_FP32}


@pytest.mark.parametrize("prec", ["fp64", "refine", "fp32"])
@pytest.mark.parametrize("distribute", [True, False])
@pytest.mark.parametrize("personal", [False, True])
def test_adjoint_matches_oracle(oracle_mod, prec, distribute, personal):
    csr = weighted_rmat(11, 8, seed=21)
    rng = np.random.default_rng(4)
    g = rng.standard_normal(csr.z)
    tele = random_teleport(csr.z, 9) if personal else None
    p, gw_o, gt_o = oracle_grads(oracle_mod, csr, g, distribute, tele)
    dg = _capi.DeviceGraph(csr)
    par = dg.params(DAMP, 1e-12, 0, False, distribute, PRECS[prec], _capi.UINT64_MAX)
    gw, gt, sweeps, st = dg.adjoint(par, p, g, tele)
    bar = 1e-4 if prec == "fp32" else 1e-9
    assert np.abs(gw - gw_o).max() <= bar * np.abs(gw_o).max()
    assert np.abs(gt - gt_o).max() <= bar * np.abs(gt_o).max()
    assert sweeps == st["fp64_sweeps"] + st["fp32_sweeps"] and sweeps > 0
    if prec != "fp64":
        assert st["fp32_sweeps"] > 0


def test_adjoint_unweighted_graph(oracle_mod):
    """Unweighted graphs: dL/dw at w = 1."""
    csr = generators.rmat_directed(10, 8, seed=5)
    g = np.random.default_rng(2).standard_normal(csr.z)
    p, gw_o, gt_o = oracle_grads(oracle_mod, csr, g, True, None)
    dg = _capi.DeviceGraph(csr)
    par = dg.params(DAMP, 1e-12, 0, False, True, _capi.NKG_PREC_FP32_REFINE, _capi.UINT64_MAX)
    gw, gt, _, _ = dg.adjoint(par, p, g)
    assert np.abs(gw - gw_o).max() <= 1e-9 * np.abs(gw_o).max()
    assert np.abs(gt - gt_o).max() <= 1e-9 * np.abs(gt_o).max()


def _with_weights(csr, w):
    return generators.InCSR(csr.z, csr.n, csr.in_ptr, csr.in_col, w,
                            np.bincount(csr.in_col, weights=w, minlength=csr.z), csr.outdeg,
                            csr.exists, csr.directed)


@pytest.mark.parametrize("distribute", [True, False])
def test_adjoint_vs_finite_differences_of_oracle(oracle_mod, distribute):
    """GPU gradients against central differences of the oracle forward."""
    csr = weighted_rmat(7, 4, seed=5)
    rng = np.random.default_rng(1)
    g = rng.standard_normal(csr.z)
    tele = random_teleport(csr.z, 3)

    def loss(c, t):
        r = oracle_mod.pagerank(c, tol=1e-15, norm=0, distribute_sinks=distribute, teleport=t,
                                max_iterations=3000)
        return float(g @ r.scores), r.scores

    _, p = loss(csr, tele)
    dg = _capi.DeviceGraph(csr)
    par = dg.params(DAMP, 1e-13, 0, False, distribute, _capi.NKG_PREC_FP32_REFINE,
                    _capi.UINT64_MAX)
    gw, gt, _, _ = dg.adjoint(par, p, g, tele)
    h = 1e-5
    for e in rng.choice(csr.arcs, 12, replace=False):
        wp = csr.in_w.copy()
        wp[e] += h
        wm = csr.in_w.copy()
        wm[e] -= h
        fd = (loss(_with_weights(csr, wp), tele)[0] - loss(_with_weights(csr, wm), tele)[0]) / (2 * h)
        assert abs(fd - gw[e]) <= 1e-7 + 1e-5 * abs(fd), (e, fd, gw[e])
    for u in rng.choice(csr.z, 6, replace=False):
        tp = tele.copy()
        tp[u] += h
        tm = tele.copy()
        tm[u] -= h
        fd = (loss(csr, tp)[0] - loss(csr, tm)[0]) / (2 * h)
        assert abs(fd - gt[u]) <= 1e-7 + 1e-5 * abs(fd), (u, fd, gt[u])


def test_adjoint_vs_gpu_finite_differences_with_set_weights():
    """Central differences (h = 1e-4) of the GPU FP64 forward, the weights
    replaced in place by nkg_graph_set_weights for every evaluation; a fixed
    400 sweeps (0.85^400 ~ 1e-28) so that both sides of a difference run the
    same arithmetic."""
    csr = weighted_rmat(14, 16, seed=11)
    rng = np.random.default_rng(7)
    g = rng.standard_normal(csr.z)
    dg = _capi.DeviceGraph(csr)
    fwd = dg.params(DAMP, 0.0, 0, False, True, _capi.NKG_PREC_FP64, 400)
    p, _, _, _ = dg.run(fwd)
    bwd = dg.params(DAMP, 1e-12, 0, False, True, _capi.NKG_PREC_FP32_REFINE, _capi.UINT64_MAX)
    gw, _, _, _ = dg.adjoint(bwd, p, g)
    h = 1e-4
    edges = rng.choice(csr.arcs, 16, replace=False)
    fds = []
    for e in edges:
        vals = []
        for sgn in (1, -1):
            w = csr.in_w.copy()
            w[e] += sgn * h
            dg.set_weights(w, np.bincount(csr.in_col, weights=w, minlength=csr.z))
            vals.append(float(g @ dg.run(fwd)[0]))
        fds.append((vals[0] - vals[1]) / (2 * h))
    fds = np.array(fds)
    scale = np.abs(gw[edges]).max()
    assert np.abs(fds - gw[edges]).max() <= 1e-5 * scale, (fds, gw[edges])


def test_set_weights_equals_fresh_graph():
    """A graph whose weights were replaced runs bit-identically to a graph
    created with the new weights (FP64 and FP32 planes, the adjoint layout
    too); weighted degrees summed on the device agree to rounding."""
    a = weighted_rmat(12, 8, seed=31)
    b = generators.with_uniform_weights(a, seed=77)
    dg = _capi.DeviceGraph(a)
    ref = _capi.DeviceGraph(b)
    g = np.random.default_rng(0).standard_normal(a.z)
    for prec in (_capi.NKG_PREC_FP64, _capi.NKG_PREC_FP32):
        dg.run(dg.params(DAMP, 1e-9, 0, False, True, prec, 200))
    p0 = dg.run(dg.params(DAMP, 1e-10, 0, False, True, _capi.NKG_PREC_FP64, 500))[0]
    bwd = dg.params(DAMP, 1e-11, 0, False, True, _capi.NKG_PREC_FP32_REFINE, _capi.UINT64_MAX)
    dg.adjoint(bwd, p0, g)  # builds the out-adjacency with the old weights
    dg.set_weights(b.in_w, b.wdeg)
    for prec in (_capi.NKG_PREC_FP64, _capi.NKG_PREC_FP32):
        par = dg.params(DAMP, 1e-9, 0, False, True, prec, 200)
        got, it, _, _ = dg.run(par)
        want, it2, _, _ = ref.run(par)
        np.testing.assert_array_equal(got, want)
        assert it == it2
    p = ref.run(dg.params(DAMP, 1e-10, 0, False, True, _capi.NKG_PREC_FP64, 500))[0]
    gw, gt, _, _ = dg.adjoint(bwd, p, g)
    gw2, gt2, _, _ = ref.adjoint(bwd, p, g)
    np.testing.assert_array_equal(gw, gw2)
    np.testing.assert_array_equal(gt, gt2)
    dg.set_weights(b.in_w)  # degrees summed on the device
    got = dg.run(dg.params(DAMP, 1e-10, 0, False, True, _capi.NKG_PREC_FP64, 500))[0]
    assert np.abs(got - p).sum() <= 1e-12


def test_run_ex_device_pointers_match_host_run():
    import torch

    csr = weighted_rmat(12, 8, seed=3)
    tele = random_teleport(csr.z, 5)
    dg = _capi.DeviceGraph(csr)
    par = dg.params(DAMP, 1e-10, 0, False, True, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
    host, it, mx, _ = dg.run(par, tele)
    dev = torch.device("cuda", 0)
    t = torch.from_numpy(tele).to(dev)
    out = torch.empty(csr.z, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    it2, mx2, _ = dg.run_ex(par, t.data_ptr(), out.data_ptr(), True)
    np.testing.assert_array_equal(out.cpu().numpy(), host)
    assert (it, mx) == (it2, mx2)
    hout = np.empty(csr.z)
    it3, _, _ = dg.run_ex(par, tele.ctypes.data, hout.ctypes.data, False)
    np.testing.assert_array_equal(hout, host)


def test_autograd_function_matches_oracle(oracle_mod):
    import torch

    from networkit_b200 import autograd

    csr = weighted_rmat(11, 8, seed=21)
    dev = torch.device("cuda", 0)
    g = np.random.default_rng(4).standard_normal(csr.z)
    tele = random_teleport(csr.z, 9)
    p_o, gw_o, gt_o = oracle_grads(oracle_mod, csr, g, True, tele)
    G = autograd.DifferentiableGraph(csr)
    w = torch.from_numpy(csr.in_w.copy()).to(dev).requires_grad_(True)
    t = torch.from_numpy(tele).to(dev).requires_grad_(True)
    scores = autograd.pagerank(G, w, t, tol=1e-12, precision="fp32_refine")
    assert np.abs(scores.detach().cpu().numpy() - p_o).sum() <= 1e-10
    loss = (scores * torch.from_numpy(g).to(dev)).sum()
    loss.backward()
    assert np.abs(w.grad.cpu().numpy() - gw_o).max() <= 1e-8 * np.abs(gw_o).max()
    assert np.abs(t.grad.cpu().numpy() - gt_o).max() <= 1e-8 * np.abs(gt_o).max()


def test_autograd_gradcheck_small_graph():
    import torch

    from networkit_b200 import autograd

    csr = weighted_rmat(4, 3, seed=8)
    dev = torch.device("cuda", 0)
    G = autograd.DifferentiableGraph(csr)
    w = torch.from_numpy(csr.in_w.copy()).to(dev).requires_grad_(True)
    t = torch.from_numpy(random_teleport(csr.z, 2)).to(dev).requires_grad_(True)

    def f(w_, t_):
        return autograd.pagerank(G, w_, t_, tol=1e-15, precision="fp64", backward_tol=1e-14,
                                 max_iterations=2000)

    assert torch.autograd.gradcheck(f, (w, t), eps=1e-6, atol=1e-8, rtol=1e-5)


def test_adjoint_rejects_bad_input():
    a = weighted_rmat(8, 4, seed=1)
    dg = _capi.DeviceGraph(a)
    z = a.z
    par = dg.params(DAMP, 1e-10, 0, True, True, _capi.NKG_PREC_FP64, 100)
    with pytest.raises(_capi.NkgError, match="normalized"):
        dg.adjoint(par, np.full(z, 1 / z), np.ones(z))
    un = _capi.DeviceGraph(generators.rmat_directed(8, 4, seed=1))
    with pytest.raises(_capi.NkgError, match="unweighted"):
        un.set_weights(np.ones(un.info()["arcs"]))
    srt = _capi.DeviceGraph(a, arc_order=1)
    par = dg.params(DAMP, 1e-10, 0, False, True, _capi.NKG_PREC_FP64, 100)
    with pytest.raises(_capi.NkgError, match="arc_order"):
        srt.adjoint(par, np.full(z, 1 / z), np.ones(z))
