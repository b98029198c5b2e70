"""Distributional parity of the GPU Monte-Carlo search with the reference's CPU
search (fixtures tests/golden/ref_search_<case>.npz, made by
make_search_golden.py from the reference's own mutate_conf / quasi_newton code
under the chain loop of its GPU kernel, monte_carlo.cu:291-348).

The random streams cannot match (Philox on the device against the reference's
host generator), so the comparison is over independent runs per ligand: the
median of the best energy found (minimum over the run's chains of the refined
energy, inter + intra at curl cap 1000, the quantity the search minimises)
must match the reference's median within 0.1 kcal/mol.  The engine makes 128
runs (128 replicas of the ligand in one batch; every chain draws from its own
Philox stream, as a separate seed would give); the reference fixtures hold
32 runs, or 128 for the broadest distributions (fast, ad4).

A median of a few dozen runs is itself uncertain: for the broadest ligands
its standard error exceeds 0.1 kcal/mol (0.14 at 32 runs for the widest).
So each case reports the difference d of the medians with its bootstrap
standard error se (both samples resampled, 2000 draws, fixed seed) and
passes when |d| <= 0.1 + 2 se: the data do not show a difference beyond the
0.1 band.  d, se and the heavy-atom RMSD of each run's best pose to the
reference's overall best pose are printed for every case.

Cases:
  vina / vinardo   plain single docking (exhaustiveness 8, heuristic steps),
                   one chain per warp and two chains per warp;
  fast             the benchmarked screen settings (Vina, exhaustiveness 128,
                   max_step 20) on the first 8 ligands of the bench's own
                   generator, at both chain widths;
  detail_vinardo   the uneven-size screen's settings (Vinardo, exhaustiveness
                   512, max_step 40);
  ad4              AutoDock 4.2 scoring (the engine's AD4 maps, read by the
                   reference's ad4cache for its run), exhaustiveness 32,
                   max_step 40.
"""
from pathlib import Path

import numpy as np
import pytest

from unidock_tools import engine, synth

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = 0.1
RUNS = 128


def median_diff(ours, theirs, draws=2000, seed=11):
    """Difference of the medians and its bootstrap standard error."""
    rng = np.random.default_rng(seed)
    d = float(np.median(ours) - np.median(theirs))
    bs = [np.median(rng.choice(ours, len(ours))) - np.median(rng.choice(theirs, len(theirs))) for _ in range(draws)]
    return d, float(np.std(bs))


def heavy_rmsd(L, heavy, pa, pb):
    a, b = L.coords(pa)[heavy], L.coords(pb)[heavy]
    return float(np.sqrt(np.mean(np.sum((a - b) ** 2, axis=1))))


_cache = {}


def load(case):
    """Fixture arrays and the engine's maps of a case (built once per module)."""
    if case not in _cache:
        path = GOLDEN / f"ref_search_{case}.npz"
        if not path.exists():
            pytest.skip(f"fixture {path.name} not generated")
        g = dict(np.load(path))
        sf = int(g.get("sf", 0))
        if "rec_xyz" in g:
            maps = engine.Maps(g["rec_xyz"], g["rec_xs"], g["center"], g["size"], float(g["spacing"]), sf=sf)
        else:
            rec = synth.make_receptor(3000, seed=int(g["rec_seed"]), with_charges=(sf == engine.SF_AD4))
            if sf == engine.SF_AD4:
                xyz, _, ad, q = engine.parse_receptor_ex(rec.to_pdbqt())
                maps = engine.Maps(xyz, ad, g["center"], g["size"], float(g["spacing"]), sf=sf, charges=q)
            else:
                maps = engine.Maps(rec.xyz, rec.xs, g["center"], g["size"], float(g["spacing"]), sf=sf)
        _cache[case] = (g, maps)
    return _cache[case]


def run_case(case, li, lanes=32, cap=0):
    g, maps = load(case)
    E = int(g["exhaustiveness"])
    max_step = int(g.get("max_step", 0))
    if "run_e" in g:
        theirs_e = g["run_e"][li]
        theirs_pose = g["run_pose"][li]
    else:
        theirs_e = g["chain_e"][li].min(axis=1)
        theirs_pose = g["chain_pose"][li][np.arange(g["chain_e"].shape[1]), g["chain_e"][li].argmin(axis=1)]
    runs = RUNS
    L = engine.Ligand(str(g["ligand_pdbqt"][li]))
    T = L.n_torsions
    assert T == int(g["n_torsions"][li])
    # same MC budget as the reference run (vina.h:191-204 heuristic, max_step cap)
    steps = 70 * 3 * (50 + L.n_atoms + 10 * (6 + T)) // 2
    if max_step > 0:
        steps = min(steps, max_step)
    assert steps == int(g["global_steps"][li])
    B = engine.Batch(maps, [L] * runs)
    B.search(exhaustiveness=E, max_step=max_step, seed=2024 + li, form=1, lanes_per_chain=lanes, bfgs_cap=cap)
    poses, e, _ = B.chains()
    e = e.reshape(runs, E)
    ours = e.min(axis=1)
    d, se = median_diff(ours, theirs_e)
    heavy = L.export()["el"] != 0
    ref_best = theirs_pose[int(np.argmin(theirs_e))][:7 + T]
    ours_best = poses.reshape(runs, E, -1)[np.arange(runs), e.argmin(axis=1), :7 + T]
    r_ours = [heavy_rmsd(L, heavy, p, ref_best) for p in ours_best]
    r_theirs = [heavy_rmsd(L, heavy, p[:7 + T], ref_best) for p in theirs_pose]
    print(f"{case} ligand {li} ({lanes} lanes, BFGS cap {cap or 'none'}): {L.n_atoms} atoms {T} torsions, "
          f"E {E}, {steps} steps, {runs} / {len(theirs_e)} runs; median best GPU {np.median(ours):.3f} reference "
          f"{np.median(theirs_e):.3f} (diff {d:+.3f}, se {se:.3f}); min GPU {ours.min():.3f} ref {theirs_e.min():.3f}; "
          f"median RMSD to reference best: GPU {np.median(r_ours):.2f} A, reference runs {np.median(r_theirs):.2f} A")
    return d, se, ours, theirs_e


def check(d, se, ours, theirs):
    assert abs(d) <= TOL + 2 * se, (d, se, np.sort(ours), np.sort(theirs))


# plain docking: every ligand with one chain per warp, two of them with two
# chains per warp (16 lanes a chain: the same random streams, another FP32
# summation order)
@pytest.mark.parametrize("case", ["vina", "vinardo"])
@pytest.mark.parametrize("li,lanes", [(0, 32), (1, 32), (2, 32), (3, 32), (0, 16), (2, 16)])
def test_best_energy_median_matches_reference(case, li, lanes):
    check(*run_case(case, li, lanes))


# the benchmarked settings: all 8 ligands at one chain per warp, half of them
# at two chains per warp
@pytest.mark.parametrize("li,lanes", [(k, 32) for k in range(8)] + [(k, 16) for k in (0, 2, 4, 7)])
def test_fast_screen_settings_match_reference(li, lanes):
    check(*run_case("fast", li, lanes))


@pytest.mark.parametrize("li", range(4))
def test_detail_vinardo_settings_match_reference(li):
    check(*run_case("detail_vinardo", li, 32))


@pytest.mark.parametrize("li", range(4))
def test_ad4_search_matches_reference(li):
    check(*run_case("ad4", li, 32))
