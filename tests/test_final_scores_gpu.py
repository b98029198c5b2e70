"""The final reported scores of a search (REMARK VINA RESULT affinity, RMSD
lower and upper bounds, INTER + INTRA, INTER, INTRA, the conf-independent part
and UNBOUND) against the reference's own post-search scoring of the same mode
poses (Vina::global_search_gpu after its search, vina.h:232-343, with
score_gpu, vina.cpp:1245-1322, called through oracle/_ref).

The engine searches, clusters, refines (refine_step 3: BFGS against the
receptor atoms) and scores on the device and host; the reference is then given
the engine's final mode poses and recomputes every reported number the way its
own CLI would: the modes ordered by their refined energies (recomputed by the
reference at those poses: the receptor-atom energy, or the maximum when a
pose's heavy atoms left the box), the intramolecular energy of the first,
conf_independent(inter + intra - that energy) per mode (AD4: inter plus the
torsional term, unbound -intra), the final order, and the RMSD bounds to the
best mode.

Bar: 1e-4 relative on the energies, 1e-3 A on lb / ub, and the same order.
Two exceptions are counted and printed, not hidden.  A mode with an atom on
a box wall (within 1e-4 A of it or outside): the receptor-atom energy adds
1e6 kcal/mol per A of distance outside the box (non_cache.cpp:35-110), so
coordinates that agree to FP32 rounding (about 1e-6 A) give inter energies
that differ by up to about a kcal/mol; refinement against a penalised box
leaves such poses, resting on the wall.  For those modes only the intra
energy is compared (and the order and RMSD bounds when the orders agree).
Second, the scoring-path energies
read the nearest-bin table (model::evali, non_cache::eval with eval_fast), so
a pair whose r^2 lies within FP32 rounding of a bin edge can fall into either
bin; the two implementations' coordinates agree to about 1e-7 relative, and
at one edge in many thousand pairs that flips one bin, a jump of at most a
few 1e-3 kcal/mol.  A difference above 1e-4 relative is accepted as such a
flip when it is below 1e-2 kcal/mol, at most once in every 20 modes.
"""
import tempfile
from pathlib import Path

import numpy as np
import pytest

from oracle import ref
from unidock_tools import engine, synth

from .conftest import BOX_CENTER, BOX_SIZE

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference build missing")]

SPACING = 0.375
HALF = 0.5 * SPACING * np.ceil(BOX_SIZE / SPACING)   # the box as the reference lays out its grid
MAXF = np.float32(np.finfo(np.float32).max)


def close(a, b, rel=1e-4):
    return abs(float(a) - float(b)) <= rel * max(1.0, abs(float(b)))


def within_box(L, pose):
    """non_cache::within (non_cache.cpp:408-418): heavy atoms in the box, margin 1e-4."""
    xyz = L.coords(pose)[L.export()["el"] != 0]
    lo, hi = BOX_CENTER - HALF - 1e-4, BOX_CENTER + HALF + 1e-4
    return bool(np.all((xyz >= lo) & (xyz <= hi)))


BIN_STEP = 1e-2
FLIPS = []
WALL = []


def on_wall(L, pose):
    """An atom (any, as non_cache scores every movable atom) within 1e-4 A of
    a box wall or outside it."""
    xyz = L.coords(pose)
    lo, hi = BOX_CENTER - HALF, BOX_CENTER + HALF
    return bool(np.any(xyz < lo + 1e-4) or np.any(xyz > hi - 1e-4))


def compare(case, L, RL, RM, modes, order_e, receptor):
    poses = np.array([p for p, _ in modes], np.float32)
    ours = np.array([en for _, en in modes], np.float32)
    rows = RL.final_scores(RM, poses, order_e, receptor)
    assert len(rows) == len(modes)
    src = rows[:, 0].astype(int)
    tie = any(close(rows[k, 1], rows[k + 1, 1]) for k in range(len(rows) - 1))
    wall = [on_wall(L, p) for p, _ in modes]
    same_order = list(src) == list(range(len(modes)))
    if not tie and not any(wall):
        assert same_order, (case, src, ours[:, 0], rows[:, 1])
    worst = 0.0
    for k, s in enumerate(src):
        o, r = ours[s], rows[k]
        # ours: affinity, lb, ub, inter+intra, inter, intra, conf-indep, unbound
        if wall[s]:
            assert close(o[5], r[6]), (case, k, o, r)
            WALL.append((case, k, float(o[4]), float(r[5])))
            if not tie and same_order:
                assert abs(o[1] - r[2]) <= 1e-3 and abs(o[2] - r[3]) <= 1e-3, (case, k, o, r)
            continue
        flipped = False
        for a, b in ((o[0], r[1]), (o[3], r[4]), (o[4], r[5]), (o[5], r[6]), (o[6], r[7]), (o[7], r[8])):
            if not close(a, b):
                assert abs(float(a) - float(b)) <= BIN_STEP, (case, k, o, r)
                flipped = True
                continue
            worst = max(worst, abs(float(a) - float(b)) / max(1.0, abs(float(b))))
        if flipped:
            FLIPS.append((case, k, o.tolist(), r.tolist()))
        if not tie and same_order:
            assert abs(o[1] - r[2]) <= 1e-3 and abs(o[2] - r[3]) <= 1e-3, (case, k, o, r)
    return worst


@pytest.fixture(scope="module")
def setup(receptor):
    with tempfile.TemporaryDirectory() as d:
        ligs, refs = [], []
        for k, l in enumerate(synth.ligand_set(6, seed=20261203, heavy=(12, 48), torsions=(0, 10))):
            txt = l.to_pdbqt()
            p = Path(d) / f"l{k}.pdbqt"
            p.write_text(txt)
            ligs.append(engine.Ligand(txt))
            refs.append((p, txt))
        yield ligs, refs, d


@pytest.mark.parametrize("sf,refine", [(engine.SF_VINA, 3), (engine.SF_VINA, 0), (engine.SF_VINARDO, 3)])
def test_final_scores_match_reference(receptor, setup, sf, refine):
    ligs, refs, d = setup
    M = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, SPACING, sf=sf)
    RM = ref.RefMaps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, SPACING, sf=sf)
    B = engine.Batch(M, ligs)
    B.search(exhaustiveness=32, max_step=20, num_modes=9, seed=77, refine_step=refine)
    worst, n = 0.0, 0
    for i, L in enumerate(ligs):
        RL = ref.RefLigand(refs[i][0], sf=sf)
        modes = B.modes(i)
        assert modes
        if refine:
            order_e = [RL.nc_eval_deriv(RM, p, 1e6, 1000.0)[0] if within_box(L, p) else MAXF for p, _ in modes]
        else:
            order_e = [RL.eval_deriv(RM, p, 1000.0, 1000.0)[0] for p, _ in modes]
        worst = max(worst, compare(f"sf {sf} refine {refine} ligand {i}", L, RL, RM, modes, order_e, refine > 0))
        n += len(modes)
    flips = [f for f in FLIPS if f[0].startswith(f"sf {sf} refine {refine} ")]
    wall = [w for w in WALL if w[0].startswith(f"sf {sf} refine {refine} ")]
    print(f"sf {sf}, refine_step {refine}: {n} modes of {len(ligs)} ligands, worst relative energy difference "
          f"{worst:.2e}; {len(flips)} mode(s) with a nearest-bin flip: {flips}; {len(wall)} mode(s) on a box wall "
          f"(case, rank, inter ours, inter reference): {wall}")
    assert len(flips) * 20 <= n


def test_final_scores_match_reference_ad4(setup):
    ligs_v, refs, d = setup
    rec = synth.make_receptor(3000, seed=1, with_charges=True)
    xyz, _, ad, q = engine.parse_receptor_ex(rec.to_pdbqt())
    M = engine.Maps(xyz, ad, BOX_CENTER, BOX_SIZE, SPACING, sf=engine.SF_AD4, charges=q)
    prefix = str(Path(d) / "rec")
    M.write(prefix)
    RM = ref.RefAd4Maps(prefix)
    texts = [l.to_pdbqt() for l in synth.ligand_set(4, seed=4242, dist="lognormal", with_charges=True)]
    ligs = [engine.Ligand(t) for t in texts]
    B = engine.Batch(M, ligs)
    B.search(exhaustiveness=16, max_step=20, num_modes=9, seed=78)
    worst = 0.0
    for i, (L, t) in enumerate(zip(ligs, texts)):
        p = Path(d) / f"ad4_{i}.pdbqt"
        p.write_text(t)
        RL = ref.RefLigand(p, sf=engine.SF_AD4)
        modes = B.modes(i)
        assert modes
        worst = max(worst, compare(f"ad4 ligand {i}", L, RL, RM, modes, None, False))
    flips = [f for f in FLIPS if f[0].startswith("ad4 ")]
    n = sum(len(B.modes(i)) for i in range(len(ligs)))
    print(f"AD4: {n} modes, worst relative energy difference {worst:.2e}; {len(flips)} mode(s) with a nearest-bin "
          f"flip: {flips}")
    assert len(flips) * 20 <= n
