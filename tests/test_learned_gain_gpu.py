"""GPU: what the trained warm-start network gains over the solve without it, on held-out cells.

The U-Net (widths 16/32/64, BF16 tensor-core convolutions) is trained on correctors that the solver itself
generates for seeded 16^3 cells of the benchmark generator, then evaluated on held-out seeds:
  - prediction: its stiffness-weighted error against the converged correctors is far below that of the untrained
    network and of the cold start u0 = 0;
  - start of the solve: the energy-optimally scaled prediction starts PCG closer to the solution in the energy
    norm of the problem than u0 = 0 (||u* - b u0||_K < ||u*||_K for every cell and case);
  - the solve itself: warm and cold starts reach the same C (within 1e-8 of max |C|, or the FP64 floor), and the
    iteration counts of both are recorded. At the 1e-9 void floor the warm start does not reduce the iterations:
    the residual rule makes PCG resolve the void's displacement, which a cold start gets from the same Krylov
    process as the solid, while the prediction's error sits in near-null modes that PCG resolves last.
"""
import numpy as np
import pytest

from oracle import density_ref as OD
from oracle import linear_ref as OL

pytestmark = pytest.mark.gpu
MAT = dict(E=1.0, nu=0.3, emin=1e-9, p=3.0)
SOLVER = dict(precision="fp64", precond="scaled", tol=1e-9, energy_tol=1e-10, maxit=4000, check_every=16)


def test_trained_network_gains_on_heldout_cells():
    import torch
    from nlfiber_b200 import learned as LN
    from nlfiber_b200 import linear as L

    n_o, n = 8, 16
    train = np.stack([OD.random_cell(10_000 + i, n_o=n_o, r=1.5, beta=16.0, kmax=2)[0] for i in range(48)])
    held = np.stack([OD.random_cell(1_000_000 + i, n_o=n_o, r=1.5, beta=16.0, kmax=2)[0] for i in range(6)])
    lh = L.LinearHomogenization((n, n, n), **MAT, **SOLVER)
    cold = lh.C_full_batched(held, want_u=True)
    tr = lh.C_full_batched(train, want_u=True)
    rho_t = torch.tensor(train, dtype=torch.float32, device="cuda")
    tgt = LN.corrector_channels(torch.from_numpy(tr["u"])).cuda()
    w = LN.loss_weights(rho_t, MAT["emin"], MAT["p"]) + 0.05
    net = LN.UNet((16, 32, 64), seed=0)
    untrained = LN.UNet((16, 32, 64), seed=0)
    LN.train(net, rho_t, tgt, w, steps=600, batch=8, lr=2e-3, seed=0)

    rho_h = torch.tensor(held, dtype=torch.float32, device="cuda")
    t_h = LN.corrector_channels(torch.from_numpy(cold["u"])).cuda()
    wh = LN.loss_weights(rho_h, MAT["emin"], MAT["p"])[..., None]

    def err(y):
        return float(torch.sqrt((wh * (y - t_h) ** 2).sum() / (wh * t_h ** 2).sum()))

    e_tr, e_un, e_0 = err(net.forward(rho_h)), err(untrained.forward(rho_h)), err(torch.zeros_like(t_h))
    assert e_tr < 0.5 * min(e_un, e_0), (e_tr, e_un, e_0)

    # the energy-optimally scaled prediction starts closer to u* in the energy norm than u0 = 0
    u0 = LN.WarmStart(net).u0(rho_h).cpu().numpy()
    oh = OL.LinearHomogenization((n, n, n), **MAT)
    for k in range(len(held)):
        s = oh.stiffness_scale(held[k])
        for I in range(6):
            us, v = cold["u"][k, I], u0[k, I]
            Kv = oh.apply_K(s, v)
            beta = float(np.sum(v * oh.apply_K(s, us)) / np.sum(v * Kv))
            d = us - beta * v
            assert np.sum(d * oh.apply_K(s, d)) < np.sum(us * oh.apply_K(s, us)), (k, I)

    # warm and cold starts give the same C; the iterations of both are recorded in the message
    warm = L.LinearHomogenization((n, n, n), **MAT, **SOLVER, scale_x0=True).C_full_batched(
        held, u0=LN.WarmStart(net).u0(rho_h))
    scale = np.abs(cold["C"]).reshape(len(held), -1).max(1)[:, None, None]
    ok = np.abs(warm["C"] - cold["C"]) <= 1e-8 * scale + 1e-13
    assert ok.all() and warm["status"] == 0, dict(cold_it=cold["it"].tolist(), warm_it=warm["it"].tolist())
    print(f"prediction error trained {e_tr:.3f} / untrained {e_un:.3f} / zero {e_0:.3f}; "
          f"iterations cold {cold['it'].tolist()} warm {warm['it'].tolist()}")
