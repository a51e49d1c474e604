"""GPU adjoint gradients against central finite differences on the adjoint
workload itself: Kronecker scale 20 (-g 20), edge weights U[0.5, 1.5], loss
weights N(0, 1), a seed-set teleport; h = 1e-6 in FP64 on 256 sampled
coordinates (128 teleport entries, 128 edge weights), each compared on its
own.

L(t, w) = sum_v loss_w[v] s[v] with s the PPR fixed point
s = (1 - d) t + d A(w) s,  A(w)[x, u] = w(u -> x) / rowsum_w(u).

Finite differences need 512 perturbed FP64 solves of a 31M-edge problem,
far beyond the CPU oracle's reach in a test, so they run on the device in
FP64 with torch's sparse products.  That operator is checked first against
the oracle's FP64 PPR (oracle.ppr_f64: 30 Jacobi sweeps from the same
start agree to 1e-12).  Each perturbed problem p is solved for its change
D = s(p) - s0 from the base fixed point s0, which satisfies
D = r(p) + d A(p) D,  r(p) = (1 - d)(t(p) - t) + d (A(p) - A) s0,
so the large common part s0 never enters a subtraction (the derivative
estimate is still the central difference of two perturbed solves:
(L(p+) - L(p-)) / 2h = loss_w . (D+ - D-) / 2h).  A(p) differs from A
only in the perturbed edge's source column, applied as a correction after
each product.  200 sweeps leave 0.85^200 < 1e-14 of D.

Tolerances, per coordinate (FP32 engine vs FP64 differences):
  teleport  |g - fd| <= 2e-5 |fd| + 2e-6 mean|fd|: the adjoint's FP32
            solution carries ~1e-6 relative rounding and the solve stops at
            an L1 change below 1e-7 of ||loss_w||_1;
  weights   |g - fd| <= 1e-4 |fd| + 4e-6 scale, scale = d s0[u] / rowsum(u)
            (|lambda[v]| + |(P lambda)[u]|): the gradient is the difference
            of those two FP32 terms, so its error follows their size, not
            the (often much smaller) difference; 4e-6 is about 60 FP32
            roundings of that size (measured on the B200: at most 7.1e-7
            of scale, teleport at most 8.8e-6 of |fd|).
"""
import numpy as np
import pytest

import oracle
from gapbs_b200 import PageRankEngine
from gapbs_b200.graph import make_graph
from conftest import gpu_available
from helpers import in_weights, row_sums, seed_teleports

pytestmark = pytest.mark.gpu

D = 0.85
H = 1e-6
SWEEPS = 200


@pytest.fixture(scope="module")
def setup():
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch
    rng = np.random.default_rng(27491095 + 3)
    g = make_graph("-g 20")
    n, m = g.num_nodes, g.num_edges_directed
    ew32 = rng.uniform(0.5, 1.5, m).astype(np.float32)
    t32 = seed_teleports(g, 1, rng, max_seeds=1024)[:, 0]
    lw32 = rng.normal(size=n).astype(np.float32)
    ew, t, lw = ew32.astype(np.float64), t32.astype(np.float64), lw32.astype(np.float64)
    rsum = row_sums(g, ew)
    win = in_weights(g, ew)
    dev = torch.device("cuda:0")
    dst_src = g.in_neighbors.astype(np.int64)
    vals = win / rsum[dst_src]
    A = torch.sparse_csr_tensor(torch.from_numpy(g.in_offsets.astype(np.int64)),
                                torch.from_numpy(dst_src), torch.from_numpy(vals),
                                size=(n, n), dtype=torch.float64).to(dev)
    return dict(torch=torch, rng=rng, g=g, n=n, m=m, ew32=ew32, t32=t32, lw32=lw32, ew=ew,
                t=t, lw=lw, rsum=rsum, win=win, A=A, dev=dev)


def test_fp64_operator_matches_oracle(setup):
    """The device FP64 operator is the oracle's PPR sweep (30 sweeps)."""
    S = setup
    torch, g, n = S["torch"], S["g"], S["n"]
    s_or, k, _ = oracle.ppr_f64(n, g.in_offsets, g.in_neighbors, g.out_offsets, S["t"],
                                in_w=S["win"], rowsum=S["rsum"], max_iters=30, epsilon=0.0)
    assert k == 30
    tt = torch.from_numpy(S["t"]).to(S["dev"])
    s = tt.clone()
    for _ in range(30):
        s = (1 - D) * tt + D * (S["A"] @ s.unsqueeze(1)).squeeze(1)
    s = s.cpu().numpy()
    assert np.max(np.abs(s - s_or)) <= 1e-12 * np.max(np.abs(s_or))


def test_adjoint_matches_central_differences(setup):
    S = setup
    torch, rng, g, n, m, dev, A = S["torch"], S["rng"], S["g"], S["n"], S["m"], S["dev"], S["A"]
    # the GPU gradients (FP32 forward, FP32 adjoint) through the C ABI
    eng = PageRankEngine(0)
    try:
        eng.upload(g, edge_w=S["ew32"])
        fwd = eng.run(100, 1e-7, teleport=S["t32"])
        gt, ge, sweeps = eng.adjoint(S["lw32"], fwd.scores, max_iters=400, epsilon=1e-7)
        assert 0 < sweeps <= 400
    finally:
        eng.close()
    gt = gt.astype(np.float64)
    ge = ge.astype(np.float64)

    tt = torch.from_numpy(S["t"]).to(dev)
    lw = torch.from_numpy(S["lw"]).to(dev)
    s0 = tt.clone()
    for _ in range(2 * SWEEPS):
        s0 = (1 - D) * tt + D * (A @ s0.unsqueeze(1)).squeeze(1)

    # teleport coordinates: r = +-(1 - d) h e_i, A unchanged
    ti = rng.choice(n, 128, replace=False)
    cols = 2 * len(ti)
    r = torch.zeros(n, cols, dtype=torch.float64, device=dev)
    idx = torch.from_numpy(ti).to(dev)
    ar = torch.arange(len(ti), device=dev)
    r[idx, 2 * ar] = (1 - D) * H
    r[idx, 2 * ar + 1] = -(1 - D) * H
    Dm = r.clone()
    for _ in range(SWEEPS):
        Dm = r + D * (A @ Dm)
    dl = lw @ Dm
    fd_t = ((dl[0::2] - dl[1::2]) / (2 * H)).cpu().numpy()

    # edge-weight coordinates: column u of A changes over u's out-row
    ei = rng.choice(m, 128, replace=False)
    out_off = g.out_offsets.astype(np.int64)
    src = np.searchsorted(out_off, ei, side="right") - 1
    rows, ccols, dvals, us = [], [], [], []
    for c, (e, u) in enumerate(zip(ei, src)):
        lo, hi = out_off[u], out_off[u + 1]
        nbr = g.out_neighbors[lo:hi].astype(np.int64)
        w = S["ew"][lo:hi]
        for sgn, col in ((1.0, 2 * c), (-1.0, 2 * c + 1)):
            w2 = w.copy()
            w2[e - lo] += sgn * H
            delta = w2 / (S["rsum"][u] + sgn * H) - w / S["rsum"][u]
            rows.append(nbr)
            ccols.append(np.full(nbr.size, col, np.int64))
            dvals.append(delta)
            us.append(np.full(nbr.size, u, np.int64))
    rows_t = torch.from_numpy(np.concatenate(rows)).to(dev)
    cols_t = torch.from_numpy(np.concatenate(ccols)).to(dev)
    dv_t = torch.from_numpy(np.concatenate(dvals)).to(dev)
    us_t = torch.from_numpy(np.concatenate(us)).to(dev)
    cols = 2 * len(ei)
    r = torch.zeros(n, cols, dtype=torch.float64, device=dev)
    r.index_put_((rows_t, cols_t), D * s0[us_t] * dv_t, accumulate=True)
    Dm = r.clone()
    for _ in range(SWEEPS):
        Y = A @ Dm
        Y.index_put_((rows_t, cols_t), Dm[us_t, cols_t] * dv_t, accumulate=True)
        Dm = r + D * Y
    dl = lw @ Dm
    fd_w = ((dl[0::2] - dl[1::2]) / (2 * H)).cpu().numpy()

    # adjoint lambda in FP64 for the edge-gradient error scale
    AT = A.to_sparse_coo().t().coalesce().to_sparse_csr()
    lam = lw.clone()
    for _ in range(2 * SWEEPS):
        lam = lw + D * (AT @ lam.unsqueeze(1)).squeeze(1)
    plam = (AT @ lam.unsqueeze(1)).squeeze(1).cpu().numpy()
    lam = lam.cpu().numpy()
    s0n = s0.cpu().numpy()

    err_t = np.abs(gt[ti] - fd_t)
    bound_t = 2e-5 * np.abs(fd_t) + 2e-6 * np.mean(np.abs(fd_t))
    v = g.out_neighbors[ei].astype(np.int64)
    scale = D * s0n[src] / S["rsum"][src] * (np.abs(lam[v]) + np.abs(plam[src]))
    err_w = np.abs(ge[ei] - fd_w)
    bound_w = 1e-4 * np.abs(fd_w) + 4e-6 * scale
    worst_t = float(np.max(err_t / bound_t))
    worst_w = float(np.max(err_w / bound_w))
    print(f"teleport: max |g-fd|/|fd| {np.max(err_t / np.maximum(np.abs(fd_t), 1e-300)):.3e}, "
          f"worst/bound {worst_t:.3f}; weights: max |g-fd|/scale "
          f"{np.max(err_w / np.maximum(scale, 1e-300)):.3e}, worst/bound {worst_w:.3f}")
    assert np.all(err_t <= bound_t), (worst_t, ti[np.argmax(err_t / bound_t)])
    assert np.all(err_w <= bound_w), (worst_w, ei[np.argmax(err_w / bound_w)])
