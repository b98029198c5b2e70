"""Distributional parity of the GPU Monte-Carlo search with the reference's CPU
search (tests/golden/ref_search_{vina,vinardo}.npz, made by make_search_golden.py
from the reference's own mutate_conf / quasi_newton code).

The random streams cannot match (Philox on the device against the reference's
host generator), so the comparison is over 32 independent runs per ligand:
the median of the best energy found (minimum over the run's 8 chains of the
refined energy, inter + intra at curl cap 1000, the quantity the search
minimises) must match the reference's median within 0.1 kcal/mol.  The 32
runs are 32 replicas of the ligand in one batch; every chain draws from its
own Philox stream, as a separate seed would give.  Heavy-atom RMSD of each
run's best pose to the reference's overall best pose is reported.  Every
ligand is searched with one chain per warp, two of them also with two chains
per warp (16 lanes each).
"""
from pathlib import Path

import numpy as np
import pytest

from unidock_tools import engine

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = [sf for sf in ("vina", "vinardo") if (GOLDEN / f"ref_search_{sf}.npz").exists()]
TOL = 0.1


def heavy_rmsd(L, heavy, pa, pb):
    a, b = L.coords(pa)[heavy], L.coords(pb)[heavy]
    return float(np.sqrt(np.mean(np.sum((a - b) ** 2, axis=1))))


@pytest.fixture(scope="module", params=CASES)
def gold(request):
    g = dict(np.load(GOLDEN / f"ref_search_{request.param}.npz"))
    sf = int(g.get("sf", 0))
    maps = engine.Maps(g["rec_xyz"], g["rec_xs"], g["center"], g["size"], float(g["spacing"]), sf=sf)
    return g, maps


# every ligand with one chain per warp; two of them with two chains per warp
# (16 lanes a chain: the same random streams, another FP32 summation order)
@pytest.mark.parametrize("li,lanes", [(0, 32), (1, 32), (2, 32), (3, 32), (0, 16), (2, 16)])
def test_best_energy_median_matches_reference(gold, li, lanes):
    g, maps = gold
    runs, E = g["chain_e"].shape[1], int(g["exhaustiveness"])
    L = engine.Ligand(str(g["ligand_pdbqt"][li]))
    T = L.n_torsions
    assert T == int(g["n_torsions"][li])
    # same MC budget as the reference run (vina.h:191-204 heuristic, no max_step cap)
    assert 70 * 3 * (50 + L.n_atoms + 10 * (6 + T)) // 2 == int(g["global_steps"][li])
    B = engine.Batch(maps, [L] * runs)
    B.search(exhaustiveness=E, max_step=0, seed=2024 + li, form=1, lanes_per_chain=lanes)
    poses, e, _ = B.chains()
    e = e.reshape(runs, E)
    ours = e.min(axis=1)
    theirs = g["chain_e"][li].min(axis=1)
    d = float(np.median(ours) - np.median(theirs))
    # poses: best of each run against the reference's overall best
    heavy = L.export()["el"] != 0
    rp = g["chain_pose"][li].reshape(runs * E, -1)[:, :7 + T]
    ref_best = rp[int(np.argmin(g["chain_e"][li].reshape(-1)))]
    ours_best = poses.reshape(runs, E, -1)[np.arange(runs), e.argmin(axis=1), :7 + T]
    theirs_best = g["chain_pose"][li][np.arange(runs), g["chain_e"][li].argmin(axis=1), :7 + T]
    r_ours = [heavy_rmsd(L, heavy, p, ref_best) for p in ours_best]
    r_theirs = [heavy_rmsd(L, heavy, p, ref_best) for p in theirs_best]
    print(f"ligand {li} ({lanes} lanes a chain): {L.n_atoms} atoms {T} torsions; median best GPU {np.median(ours):.3f} "
          f"reference {np.median(theirs):.3f} (diff {d:+.3f}); min GPU {ours.min():.3f} ref {theirs.min():.3f}; "
          f"median RMSD to reference best: GPU {np.median(r_ours):.2f} A, reference runs {np.median(r_theirs):.2f} A")
    assert abs(d) <= TOL, (np.sort(ours), np.sort(theirs))
