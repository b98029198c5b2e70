"""GPU local optimisation (ud_optimize, the quasi_newton path) against the
oracle's BFGS restatement from the same starting poses, and fixed-pose
energies/gradients against the committed reference golden vectors, for the
Vina and Vinardo scoring functions."""
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import Oracle
from unidock_tools import engine

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module", params=["vina", "vinardo"])
def setup(request):
    gold = dict(np.load(GOLDEN / f"ref_{request.param}_small.npz"))
    gold["sf"] = int(gold["sf"])
    maps = engine.Maps(gold["rec_xyz"], gold["rec_xs"], gold["center"], gold["size"], float(gold["spacing"]),
                       types=gold["types"], sf=gold["sf"])
    ligs = [engine.Ligand(str(t)) for t in gold["ligand_pdbqt"]]
    batch = engine.Batch(maps, ligs)
    return gold, maps, ligs, batch


def test_energies_match_golden(setup):
    gold, maps, ligs, batch = setup
    stride = 7 + batch.max_torsions
    for li, L in enumerate(ligs):
        T = L.n_torsions
        P = np.zeros((gold["poses"].shape[1], stride), np.float32)
        P[:, :7 + T] = gold["poses"][li, :, :7 + T]
        for v, E, G in ((1000.0, gold["e1000"], gold["g1000"]), (10.0, gold["e10"], gold["g10"])):
            e, g = batch.score_grad(np.full(len(P), li), P, v, v)
            for k in range(len(P)):
                assert abs(e[k] - E[li, k]) <= 1e-4 * max(1.0, abs(E[li, k])), (li, k, e[k], E[li, k])
                gr = G[li, k, :6 + T]
                assert np.linalg.norm(g[k, :6 + T] - gr) <= 1e-4 * max(1.0, np.linalg.norm(gr))


def test_bfgs_matches_oracle_from_same_start(setup):
    gold, maps, ligs, batch = setup
    o = Oracle(np.float32)
    fast, smooth = o.tables(sf=gold["sf"])
    om = o.maps(gold["rec_xyz"], gold["rec_xs"], gold["dims"], gold["init"], gold["factor_inv"], gold["types"],
                sf=gold["sf"])
    grid = o.grid(om, gold["dims"], gold["init"], gold["factor"], gold["factor_inv"])
    sm = {int(t): k for k, t in enumerate(gold["types"])}
    stride = 7 + batch.max_torsions
    close, total, improved = 0, 0, 0
    eg, eor = [], []
    for li, L in enumerate(ligs):
        T = L.n_torsions
        P = np.zeros((gold["poses"].shape[1], stride), np.float32)
        P[:, :7 + T] = gold["poses"][li, :, :7 + T]
        e0, _ = batch.score_grad(np.full(len(P), li), P, 10.0, 10.0)
        out, e, ev = batch.optimize(np.full(len(P), li), P, v=10.0, max_steps=20)
        ol = o.ligand(L.export(), sm)
        for k in range(len(P)):
            eo, _, _ = o.bfgs(ol, grid, smooth, P[k, :7 + T], 20, 10.0)
            total += 1
            close += abs(e[k] - eo) <= 1e-3 * max(1.0, abs(eo))
            improved += e[k] <= e0[k] + 1e-5
            eg.append(e[k])
            eor.append(eo)
        # the returned energy is the energy of the returned pose
        e_chk, _ = batch.score_grad(np.full(len(P), li), out, 10.0, 10.0)
        np.testing.assert_allclose(e_chk, e, rtol=1e-4, atol=1e-4)
    assert improved == total
    # Both are FP32 BFGS runs from the same start; a line search can branch on
    # last-bit differences (contracted multiply-adds, reassociated sums), after
    # which the two runs reach different nearby minima.  Most runs must agree
    # and the GPU's final energies must be no worse on average.
    eg, eor = np.array(eg), np.array(eor)
    print("bfgs gpu-oracle diffs:", np.round(eg - eor, 4).tolist())
    assert close >= 0.5 * total, (close, total)
    assert eg.mean() <= eor.mean() + 0.05 * np.abs(eor).mean() + 1e-3, (eg.mean(), eor.mean())
