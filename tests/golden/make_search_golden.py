"""Generate tests/golden/ref_search_<sf>.npz: the reference's own CPU Monte-Carlo
search (oracle/_ref/libudref.so, the reference's mutate_conf / quasi_newton /
output container under the chain loop of monte_carlo.cu:2319-2356) run with
32 seeds on seeded synthetic ligands, as the distribution the GPU search is
compared against.

Settings follow the plain single-docking case: Vina (or Vinardo), exhaustiveness 8, the
heuristic global step count min(70*3*(50 + N + 10*(6 + T))/2, max_step) with no
max_step cap (unidock/src/lib/vina.h:191-204), per-ligand BFGS steps
(25 + N)/3, curl cap 10 during the search and 1000 for the refinement of
improved poses.  Receptor: 3000 synthetic atoms, 22.5 A box at 0.375 A.

Stored per ligand and seed: every chain's best energy (inter + intra at curl
cap 1000, the quantity the search minimises) and best pose.

Run:  python tests/golden/make_search_golden.py [vina|vinardo]   (about 10 minutes on 8 threads)
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
EXHAUSTIVENESS = 8
BOX = 22.5
SPACING = 0.375
# (heavy atoms, torsions, generator seed): the plain-docking ligand (24 / 6) and
# three sizes from the batched-screen range
LIGANDS = [(24, 6, 31), (16, 2, 32), (32, 8, 33), (40, 10, 34)]


def global_steps(n_atoms, n_torsions):
    return 70 * 3 * (50 + n_atoms + 10 * (6 + n_torsions)) // 2


def main(name="vina"):
    sf = {"vina": 0, "vinardo": 2}[name]
    threads = os.cpu_count()
    rec = synth.make_receptor(3000, seed=1)
    center = np.zeros(3, np.float32)
    size = np.full(3, BOX, np.float32)
    R = ref.RefMaps(rec.xyz, rec.xs, center, size, SPACING, sf=sf)
    texts, energies, poses, gsteps, n_tors = [], [], [], [], []
    max_t = max(t for _, t, _ in LIGANDS)
    with tempfile.TemporaryDirectory() as d:
        for k, (nh, nt, s) in enumerate(LIGANDS):
            txt = synth.make_ligand(nh, nt, seed=s).to_pdbqt()
            p = Path(d) / f"l{k}.pdbqt"
            p.write_text(txt)
            RL = ref.RefLigand(p, sf=sf)
            gs = global_steps(RL.n_atoms, RL.n_torsions)
            t0 = time.perf_counter()
            e_l, p_l = [], []
            for seed in range(SEEDS):
                be, bp, _ = RL.mc(R, 1000 + seed, EXHAUSTIVENESS, gs, None, threads)
                e_l.append(be)
                p_l.append(np.pad(bp, ((0, 0), (0, max_t - RL.n_torsions))))
            print(f"ligand {k}: {RL.n_atoms} atoms, {RL.n_torsions} torsions, {gs} steps, "
                  f"median best {np.median(np.min(e_l, axis=1)):.3f}, {time.perf_counter() - t0:.0f} s", flush=True)
            texts.append(txt)
            energies.append(e_l)
            poses.append(p_l)
            gsteps.append(gs)
            n_tors.append(RL.n_torsions)
    out = ROOT / "tests" / "golden" / f"ref_search_{name}.npz"
    np.savez_compressed(out, sf=np.int32(sf), rec_xyz=rec.xyz, rec_xs=rec.xs, center=center, size=size, spacing=np.float32(SPACING),
                        ligand_pdbqt=np.array(texts), n_torsions=np.array(n_tors, np.int32),
                        global_steps=np.array(gsteps, np.int32), exhaustiveness=np.int32(EXHAUSTIVENESS),
                        chain_e=np.array(energies, np.float32), chain_pose=np.array(poses, np.float32),
                        threads=np.int32(threads))
    print("wrote", out, out.stat().st_size, "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "vina")
