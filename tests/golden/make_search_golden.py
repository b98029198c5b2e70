"""Generate tests/golden/ref_search_<case>.npz: the reference's own CPU Monte-Carlo
search (oracle/_ref/libudref.so, the reference's mutate_conf / quasi_newton
code under the chain loop of its GPU kernel, monte_carlo.cu:291-348) run with
32 seeds on seeded synthetic ligands, as the distribution the GPU search is
compared against.

Cases:
  vina, vinardo    the plain single-docking settings: exhaustiveness 8, the
                   heuristic global step count min(70*3*(50 + N + 10*(6 + T))/2,
                   max_step) with no max_step cap (unidock/src/lib/vina.h:191-204),
                   four hand-picked ligand sizes.  Every chain's best energy and
                   pose are stored.
  fast             the benchmarked batched-screen settings: Vina, search_mode
                   fast (exhaustiveness 128, max_step 20), the first 8 ligands of
                   the screen's generator (U{12..48} heavy atoms, U{0..10}
                   torsions, seed 20261203).
  detail_vinardo   the uneven-size screen: Vinardo, search_mode detail
                   (exhaustiveness 512, max_step 40), the first 4 ligands of its
                   generator (lognormal sizes, median 28 heavy atoms, seed 8192).
  ad4              AutoDock 4.2 scoring: the GPU engine's AD4 maps (written as
                   AutoGrid .map files and read back by the reference's
                   ad4cache), ligands with partial charges, exhaustiveness 32,
                   max_step 40.  Needs a GPU (the maps are built by the engine).
For the three named batched cases each run's best energy and best pose are
stored (run_e, run_pose); fast and ad4 have 128 runs per ligand (their
broadest distributions need them for a precise median), the others 32.

Run r seeds its chains 1000 + 65536 r + k (k the chain), so that no two chains
of any runs share a random stream and the 32 runs are independent.

All cases: per-ligand BFGS steps (25 + N)/3, curl cap 10 during the search and
1000 for the refinement of improved poses; receptor 3000 synthetic atoms, 22.5 A
box at 0.375 A.

Run:  python tests/golden/make_search_golden.py <case>
(fast: about 10 minutes on 8 threads; detail_vinardo: about 40.)
"""
import os
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "uni-dock_b200"))

from oracle import ref  # noqa: E402
from unidock_tools import synth  # noqa: E402

SEEDS = 32
BOX = 22.5
SPACING = 0.375
# (heavy atoms, torsions, generator seed) of the plain-docking cases: the
# plain-docking ligand (24 / 6) and three sizes from the batched-screen range
HAND_PICKED = [(24, 6, 31), (16, 2, 32), (32, 8, 33), (40, 10, 34)]
CASES = {
    "vina": dict(sf=0, exhaustiveness=8, max_step=0),
    "vinardo": dict(sf=2, exhaustiveness=8, max_step=0),
    "fast": dict(sf=0, exhaustiveness=128, max_step=20, n=8, seed=20261203, dist="uniform", runs=128),
    "detail_vinardo": dict(sf=2, exhaustiveness=512, max_step=40, n=4, seed=8192, dist="lognormal"),
    "ad4": dict(sf=1, exhaustiveness=32, max_step=40, n=4, seed=4242, dist="lognormal", runs=128),
}


def global_steps(n_atoms, n_torsions, max_step):
    g = 70 * 3 * (50 + n_atoms + 10 * (6 + n_torsions)) // 2
    return min(g, max_step) if max_step > 0 else g


def case_ligands(name):
    c = CASES[name]
    if "n" not in c:
        return [synth.make_ligand(nh, nt, seed=s) for nh, nt, s in HAND_PICKED]
    return synth.ligand_set(c["n"], seed=c["seed"], dist=c["dist"], with_charges=(c["sf"] == 1))


def ad4_maps(rec, center, size, d):
    """The engine's AD4 maps for `rec` written as AutoGrid files under d and
    read back by the reference's ad4cache (the engine is the map producer
    here, as autogrid4 is for the reference)."""
    from unidock_tools import engine
    xyz, _, ad, q = engine.parse_receptor_ex(rec.to_pdbqt())
    m = engine.Maps(xyz, ad, center, size, SPACING, sf=engine.SF_AD4, charges=q)
    prefix = str(Path(d) / "rec")
    m.write(prefix)
    return ref.RefAd4Maps(prefix)


def main(name):
    c = CASES[name]
    sf, E = c["sf"], c["exhaustiveness"]
    threads = os.cpu_count()
    rec = synth.make_receptor(3000, seed=1, with_charges=(sf == 1))
    center = np.zeros(3, np.float32)
    size = np.full(3, BOX, np.float32)
    ligs = case_ligands(name)
    texts, energies, poses, gsteps, n_tors = [], [], [], [], []
    max_t = max(L.n_torsions for L in ligs)
    with tempfile.TemporaryDirectory() as d:
        R = ad4_maps(rec, center, size, d) if sf == 1 else ref.RefMaps(rec.xyz, rec.xs, center, size, SPACING, sf=sf)
        for k, L in enumerate(ligs):
            txt = L.to_pdbqt()
            p = Path(d) / f"l{k}.pdbqt"
            p.write_text(txt)
            RL = ref.RefLigand(p, sf=sf)
            gs = global_steps(RL.n_atoms, RL.n_torsions, c["max_step"])
            t0 = time.perf_counter()
            e_l, p_l = [], []
            for seed in range(c.get("runs", SEEDS)):
                # chain k of a run draws from the generator seeded run_seed + k,
                # so run seeds 65536 apart keep every chain's stream distinct
                be, bp, _ = RL.mc(R, 1000 + 65536 * seed, E, gs, None, threads)
                if "n" in c:  # the run's best chain only
                    i = int(np.argmin(be))
                    e_l.append(be[i])
                    p_l.append(np.pad(bp[i], (0, max_t - RL.n_torsions)))
                else:
                    e_l.append(be)
                    p_l.append(np.pad(bp, ((0, 0), (0, max_t - RL.n_torsions))))
            best = [float(np.min(e)) for e in e_l]
            print(f"ligand {k}: {RL.n_atoms} atoms, {RL.n_torsions} torsions, {gs} steps, "
                  f"median best {np.median(best):.3f}, {time.perf_counter() - t0:.0f} s", flush=True)
            texts.append(txt)
            energies.append(e_l)
            poses.append(p_l)
            gsteps.append(gs)
            n_tors.append(RL.n_torsions)
    out = Path(os.environ.get("UD_GOLDEN_OUT", ROOT / "tests" / "golden")) / f"ref_search_{name}.npz"
    common = dict(sf=np.int32(sf), rec_seed=np.int32(1), center=center, size=size, spacing=np.float32(SPACING),
                  ligand_pdbqt=np.array(texts), n_torsions=np.array(n_tors, np.int32),
                  global_steps=np.array(gsteps, np.int32), exhaustiveness=np.int32(E),
                  max_step=np.int32(c["max_step"]), threads=np.int32(threads))
    if "n" in c:
        np.savez_compressed(out, run_e=np.array(energies, np.float32), run_pose=np.array(poses, np.float32),
                            **common)
    else:
        np.savez_compressed(out, rec_xyz=rec.xyz, rec_xs=rec.xs, chain_e=np.array(energies, np.float32),
                            chain_pose=np.array(poses, np.float32), **common)
    print("wrote", out, out.stat().st_size, "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "vina")
