"""Generate the golden fixtures of tests/golden/ from the reference's own CPU
code (oracle/_ref/libudref.so, built by oracle/Makefile from the reference
sources).  The reference's tests pin no energies, gradients or maps, so these
vectors are produced here on seeded synthetic inputs:

  ref_vina_small.npz     receptor + 12 A box maps (sampled points), 4 ligands
                         (PDBQT text), 8 poses each, reference eval_deriv
                         energies and gradients at curl caps 1000 and 10,
                         scoring energies, and sampled type-pair table values,
                         Vina scoring function with its default weights.
  ref_vinardo_small.npz  the same inputs scored with Vinardo.

Run:  python tests/golden/make_golden.py [vina|vinardo|all]
"""
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "uni-dock_b200"))

from oracle import ref  # noqa: E402
from unidock_tools import synth  # noqa: E402

TYPES = [0, 1, 2, 3, 4, 5, 8, 9, 10, 12, 13]


SF_NAMES = {"vina": 0, "vinardo": 2}


def make(name):
    sf = SF_NAMES[name]
    rng = np.random.default_rng(2026)
    rec = synth.make_receptor(1200, radius=30.0, seed=11)
    center = np.zeros(3, np.float32)
    size = np.full(3, 12.0, np.float32)
    R = ref.RefMaps(rec.xyz, rec.xs, center, size, 0.375, sf=sf, types=TYPES)
    dims = R.dims.copy()
    npts = int(dims.prod())
    sample_idx = np.sort(rng.choice(npts, 3000, replace=False)).astype(np.int64)
    map_samples = np.stack([R.get(t).reshape(-1)[sample_idx] for t in TYPES])

    ligs, texts = [], []
    with tempfile.TemporaryDirectory() as d:
        for k, (nh, nt) in enumerate([(14, 2), (22, 5), (31, 8), (40, 10)]):
            L = synth.make_ligand(nh, nt, seed=4242 + k)
            txt = L.to_pdbqt()
            p = Path(d) / f"l{k}.pdbqt"
            p.write_text(txt)
            texts.append(txt)
            ligs.append(ref.RefLigand(p, sf=sf))
        poses, e1000, g1000, e10, g10, score = [], [], [], [], [], []
        for k, RL in enumerate(ligs):
            P = synth.random_poses(8, RL.n_torsions, -3.0, 3.0, seed=77 + k)
            pk, e1k, g1k, e10k, g10k, sk = [], [], [], [], [], []
            for pose in P:
                e, g, _ = RL.eval_deriv(R, pose, 1000.0, 1000.0)
                ea, ga, _ = RL.eval_deriv(R, pose, 10.0, 10.0)
                sc = RL.score(R, pose, 1000.0)
                pk.append(np.pad(pose, (0, 10 - RL.n_torsions)))
                e1k.append(e); g1k.append(np.pad(g, (0, 10 - RL.n_torsions)))
                e10k.append(ea); g10k.append(np.pad(ga, (0, 10 - RL.n_torsions)))
                sk.append(sc)
            poses.append(pk); e1000.append(e1k); g1000.append(g1k); e10.append(e10k); g10.append(g10k)
            score.append(sk)
        # type-pair table samples (precalculate::eval_fast)
        t1 = rng.integers(0, 19, 400)
        t2 = rng.integers(0, 19, 400)
        r2 = rng.uniform(0.0, 63.9, 400).astype(np.float32)
        fast = np.array([ref.lib().udref_table_fast(R.h, int(a), int(b), float(c)) for a, b, c in zip(t1, t2, r2)],
                        np.float32)
        ntors = np.array([RL.n_torsions for RL in ligs], np.int32)
    out = ROOT / "tests" / "golden" / f"ref_{name}_small.npz"
    np.savez_compressed(
        out, rec_xyz=rec.xyz, rec_xs=rec.xs, center=center, size=size, spacing=np.float32(0.375),
        types=np.array(TYPES, np.int32), dims=dims, init=R.init, factor=R.factor, factor_inv=R.factor_inv,
        sample_idx=sample_idx, map_samples=map_samples, ligand_pdbqt=np.array(texts), n_torsions=ntors,
        poses=np.array(poses, np.float32), e1000=np.array(e1000, np.float32), g1000=np.array(g1000, np.float32),
        e10=np.array(e10, np.float32), g10=np.array(g10, np.float32), score=np.array(score, np.float32),
        sf=np.int32(sf), tab_t1=t1.astype(np.int32), tab_t2=t2.astype(np.int32), tab_r2=r2, tab_fast=fast)
    print("wrote", out, out.stat().st_size, "bytes")


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "all"
    for nm in (SF_NAMES if which == "all" else [which]):
        make(nm)
