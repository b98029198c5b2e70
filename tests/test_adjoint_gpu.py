"""Adjoint kernel (ud_score_adjoint) and the torch.autograd binding.

  * reference mode: energies and pose gradients equal the reference's
    model::eval_deriv (FP32 CPU) within 1e-4 relative, the torque mapped to the
    quaternion gradient 2 (0, tau) (x) q;
  * exact mode: pose gradients within 1e-4 relative of FP64 central
    differences (h = 1e-5, quaternion renormalised) of the FP64 oracle's
    energy, and term-weight gradients within 1e-4 relative of FP64 central
    differences over the weights (maps and tables rebuilt at w +- h).  The
    energy is piecewise smooth (trilinear cells, r^2 table bins); where a kink
    lies within +-h of a pose the h = 1e-5 difference quotient straddles it,
    which shows as disagreement with h = 1e-6, and that pose is checked
    against h = 1e-6 instead (counted and printed);
  * ud_maps_set_weights equals maps built with the same weights;
  * autograd: gradients of docking_energy equal the adjoint's.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import ref
from oracle.oracle import Oracle, VINA_W
from unidock_tools import engine

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden" / "ref_vina_small.npz"
REL = 1e-4


@pytest.fixture(scope="module")
def setup():
    gold = dict(np.load(GOLD))
    maps = engine.Maps(gold["rec_xyz"], gold["rec_xs"], gold["center"], gold["size"], float(gold["spacing"]),
                       types=gold["types"])
    ligs = [engine.Ligand(str(t)) for t in gold["ligand_pdbqt"]]
    batch = engine.Batch(maps, ligs)
    return gold, maps, ligs, batch


@pytest.fixture(scope="module")
def o64(setup):
    gold = setup[0]
    o = Oracle(np.float64)
    sm = {int(t): k for k, t in enumerate(gold["types"])}
    ligs = [o.ligand(engine.Ligand(str(t)).export(), sm) for t in gold["ligand_pdbqt"]]

    def model(weights):
        fast, smooth = o.tables(weights=weights)
        mp = o.maps(gold["rec_xyz"], gold["rec_xs"], gold["dims"], gold["init"], gold["factor_inv"], gold["types"],
                    weights=weights)
        grid = o.grid(mp, gold["dims"], gold["init"], gold["factor"], gold["factor_inv"])
        return smooth, grid

    return o, ligs, model


def quat_grad(tau, q):
    """2 (0, tau) (x) q: the gradient over q of a left-applied rotation with torque tau."""
    q0, qv = q[0], q[1:]
    return np.concatenate([[-2.0 * np.dot(tau, qv)], 2.0 * (q0 * tau + np.cross(tau, qv))])


def padded(gold, li, ligs, stride):
    T = ligs[li].n_torsions
    P = np.zeros((gold["poses"].shape[1], stride), np.float32)
    P[:, :7 + T] = gold["poses"][li, :, :7 + T]
    return P


@pytest.mark.parametrize("v", [1000.0, 10.0])
def test_reference_mode_matches_reference_eval_deriv(setup, v):
    gold, maps, ligs, B = setup
    stride = 7 + B.max_torsions
    for li, L in enumerate(ligs):
        T = L.n_torsions
        P = padded(gold, li, ligs, stride)
        e, g, _ = B.score_adjoint(np.full(len(P), li), P, v, v, exact=False, weights_grad=False)
        e_sg, g_sg = B.score_grad(np.full(len(P), li), P, v, v)
        np.testing.assert_array_equal(e, e_sg)        # same evaluation as the BFGS path
        E = gold["e1000"] if v == 1000.0 else gold["e10"]
        G = gold["g1000"] if v == 1000.0 else gold["g10"]
        for k in range(len(P)):
            er, gr = float(E[li, k]), G[li, k, :6 + T].astype(np.float64)
            assert abs(e[k] - er) <= REL * max(1.0, abs(er))
            want = np.concatenate([gr[:3], quat_grad(gr[3:6], P[k, 3:7].astype(np.float64)), gr[6:]])
            assert np.linalg.norm(g[k, :7 + T] - want) <= REL * max(1.0, np.linalg.norm(want)), (li, k)


def fd_pose(o, L, smooth, grid, pose, v, h=1e-5):
    pose = pose.astype(np.float64)
    out = np.zeros(len(pose))
    for j in range(len(pose)):
        ev = []
        for sgn in (1.0, -1.0):
            p = pose.copy()
            p[j] += sgn * h
            p[3:7] /= np.linalg.norm(p[3:7])
            ev.append(o.eval_deriv(L, grid, smooth, p, v, v)[0])
        out[j] = (ev[0] - ev[1]) / (2 * h)
    return out


@pytest.mark.parametrize("v", [1000.0, 10.0])
def test_exact_mode_matches_fp64_central_differences(setup, o64, v):
    gold, maps, ligs, B = setup
    o, oligs, model = o64
    smooth, grid = model(VINA_W)
    stride = 7 + B.max_torsions
    errs, near_kink = [], 0
    for li, L in enumerate(ligs):
        T = L.n_torsions
        P = padded(gold, li, ligs, stride)
        e, g, _ = B.score_adjoint(np.full(len(P), li), P, v, v, exact=True, weights_grad=False)
        for k in range(len(P)):
            fd = fd_pose(o, oligs[li], smooth, grid, P[k, :7 + T], v)
            fd_small = fd_pose(o, oligs[li], smooth, grid, P[k, :7 + T], v, h=1e-6)
            if np.linalg.norm(fd - fd_small) > 1e-5 * max(1.0, np.linalg.norm(fd_small)):
                near_kink += 1
                fd = fd_small
            err = np.linalg.norm(g[k, :7 + T] - fd) / max(1.0, np.linalg.norm(fd))
            errs.append(err)
            assert err <= REL, (li, k, err, g[k, :7 + T], fd)
    print(f"pose gradient vs FP64 FD (v={v}): max rel {max(errs):.3g} median {float(np.median(errs)):.3g}, "
          f"{near_kink} of {len(errs)} poses within h of a kink (checked at h=1e-6)")


def test_weight_gradient_matches_fp64_central_differences(setup, o64):
    gold, maps, ligs, B = setup
    o, oligs, model = o64
    nt = maps.n_terms
    assert nt == 6
    stride = 7 + B.max_torsions
    sel = [(li, k) for li in range(len(ligs)) for k in (0, 3)]
    lig_of = np.array([li for li, _ in sel])
    P = np.stack([padded(gold, li, ligs, stride)[k] for li, k in sel])
    _, _, dw = B.score_adjoint(lig_of, P, 1000.0, 1000.0, exact=True)
    h = 1e-3
    fd = np.zeros((len(sel), nt))
    for t in range(nt):
        ev = []
        for sgn in (1.0, -1.0):
            w = VINA_W.copy()
            w[t] += sgn * h
            smooth, grid = model(w)
            ev.append([o.eval_deriv(oligs[li], grid, smooth, P[i, :7 + ligs[li].n_torsions].astype(np.float64))[0]
                       for i, (li, _) in enumerate(sel)])
        fd[:, t] = (np.array(ev[0]) - np.array(ev[1])) / (2 * h)
    for i in range(len(sel)):
        assert np.linalg.norm(dw[i] - fd[i]) <= REL * max(1.0, np.linalg.norm(fd[i])), (sel[i], dw[i], fd[i])


def test_set_weights_equals_maps_built_with_weights(setup):
    gold, maps, ligs, B = setup
    rng = np.random.default_rng(5)
    w0 = maps.weights()
    w2 = (w0 * rng.uniform(0.8, 1.2, size=w0.shape)).astype(np.float32)
    m2 = engine.Maps(gold["rec_xyz"], gold["rec_xs"], gold["center"], gold["size"], float(gold["spacing"]),
                     types=gold["types"], weights=np.concatenate([w2, [0.05846]]).astype(np.float32))
    mw = engine.Maps(gold["rec_xyz"], gold["rec_xs"], gold["center"], gold["size"], float(gold["spacing"]),
                     types=gold["types"])
    mw.set_weights(w2)
    np.testing.assert_array_equal(mw.weights(), w2)
    for t in gold["types"]:
        a, b = mw.read(int(t)), m2.read(int(t))
        assert np.abs(a - b).max() <= 1e-5 * max(1.0, np.abs(b).max()), int(t)
    b2, bw = engine.Batch(m2, ligs), engine.Batch(mw, ligs)
    stride = 7 + B.max_torsions
    for li in range(len(ligs)):
        P = padded(gold, li, ligs, stride)
        e2, g2 = b2.score_grad(np.full(len(P), li), P)
        ew, gw = bw.score_grad(np.full(len(P), li), P)
        np.testing.assert_allclose(ew, e2, rtol=REL, atol=REL)
        np.testing.assert_allclose(gw, g2, rtol=1e-3, atol=REL * max(1.0, np.abs(g2).max()))


def test_autograd_matches_adjoint(setup):
    import torch
    from unidock_tools.autograd import docking_energy
    gold, _, ligs, _ = setup
    maps = engine.Maps(gold["rec_xyz"], gold["rec_xs"], gold["center"], gold["size"], float(gold["spacing"]),
                       types=gold["types"])
    B = engine.Batch(maps, ligs)
    stride = 7 + B.max_torsions
    P = np.concatenate([padded(gold, li, ligs, stride) for li in range(len(ligs))])
    lig_of = np.repeat(np.arange(len(ligs)), gold["poses"].shape[1])
    e_ref, g_ref, dw_ref = B.score_adjoint(lig_of, P, exact=True)
    poses = torch.tensor(P, device="cuda", requires_grad=True)
    w = torch.tensor(maps.weights(), device="cuda", requires_grad=True)
    E = docking_energy(B, torch.tensor(lig_of, device="cuda"), poses, w)
    # the Function renormalises q (last-bit changes of unit quaternions)
    np.testing.assert_allclose(E.detach().cpu().numpy(), e_ref, rtol=1e-5, atol=1e-5)
    E.sum().backward()
    np.testing.assert_allclose(poses.grad.cpu().numpy(), g_ref, rtol=1e-5, atol=1e-5 * np.abs(g_ref).max())
    np.testing.assert_allclose(w.grad.cpu().numpy(), dw_ref.sum(0), rtol=1e-5)
    # new weights through the Function: energies follow maps built with them
    w2 = (w.detach() * 1.1).requires_grad_(True)
    E2 = docking_energy(B, torch.tensor(lig_of, device="cuda"), poses.detach(), w2)
    m2 = engine.Maps(gold["rec_xyz"], gold["rec_xs"], gold["center"], gold["size"], float(gold["spacing"]),
                     types=gold["types"],
                     weights=np.concatenate([w2.detach().cpu().numpy(), [0.05846]]).astype(np.float32))
    e2, _, _ = engine.Batch(m2, ligs).score_adjoint(lig_of, P, exact=True, weights_grad=False)
    np.testing.assert_allclose(E2.detach().cpu().numpy(), e2, rtol=REL, atol=REL)
