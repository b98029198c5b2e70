"""Fixed-pose energy and pose gradient (model::eval_deriv) on the GPU against the
reference's FP32 CPU path, at seeded random poses; tolerance 1e-4 relative."""
import numpy as np
import pytest

from oracle import ref
from unidock_tools import engine, synth

from .conftest import BOX_CENTER, BOX_SIZE

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference build missing")]

REL = 1e-4


@pytest.fixture(scope="module")
def setup(receptor, tmp_path_factory):
    d = tmp_path_factory.mktemp("score")
    ligs, refs = [], []
    for k in range(6):
        L = synth.make_ligand(12 + 7 * k, min(k * 2, 10), seed=500 + k)
        txt = L.to_pdbqt()
        p = d / f"l{k}.pdbqt"
        p.write_text(txt)
        ligs.append(engine.Ligand(txt))
        refs.append(ref.RefLigand(p))
    M = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    R = ref.RefMaps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    B = engine.Batch(M, ligs)
    return ligs, refs, M, R, B


def poses_for(lig, n, seed, lo=-8.0, hi=8.0):
    return synth.random_poses(n, lig.n_torsions, lo, hi, seed)


@pytest.mark.parametrize("v", [1000.0, 10.0])
def test_energy_and_gradient_match_reference(setup, v):
    ligs, refs, M, R, B = setup
    stride = 7 + B.max_torsions
    for li, (L, RL) in enumerate(zip(ligs, refs)):
        P = poses_for(L, 16, seed=li + int(v))
        full = np.zeros((len(P), stride), np.float32)
        full[:, :P.shape[1]] = P
        e, g = B.score_grad(np.full(len(P), li), full, v, v)
        for k in range(len(P)):
            er, gr, _ = RL.eval_deriv(R, P[k], v, v)
            assert abs(e[k] - er) <= REL * max(1.0, abs(er)), (li, k, e[k], er)
            gk = g[k, :6 + L.n_torsions]
            assert np.linalg.norm(gk - gr) <= REL * max(1.0, np.linalg.norm(gr)), (li, k, gk, gr)


def test_out_of_box_penalty(setup):
    ligs, refs, M, R, B = setup
    stride = 7 + B.max_torsions
    L, RL = ligs[2], refs[2]
    P = poses_for(L, 8, seed=9, lo=14.0, hi=20.0)  # partly outside the 22.5 A box
    full = np.zeros((len(P), stride), np.float32)
    full[:, :P.shape[1]] = P
    e, g = B.score_grad(np.full(len(P), 2), full)
    for k in range(len(P)):
        er, gr, _ = RL.eval_deriv(R, P[k])
        assert abs(e[k] - er) <= REL * max(1.0, abs(er))
        assert np.linalg.norm(g[k, :6 + L.n_torsions] - gr) <= REL * max(1.0, np.linalg.norm(gr))


def test_scoring_energies_match_reference(setup):
    ligs, refs, M, R, B = setup
    stride = 7 + B.max_torsions
    for li, (L, RL) in enumerate(zip(ligs, refs)):
        P = poses_for(L, 8, seed=77 + li, lo=-5.0, hi=5.0)
        full = np.zeros((len(P), stride), np.float32)
        full[:, :P.shape[1]] = P
        out = B.score(np.full(len(P), li), full, 1000.0)
        for k in range(len(P)):
            r = RL.score(R, P[k], 1000.0)
            assert abs(out[k, 0] - r[0]) <= REL * max(1.0, abs(r[0]))
            assert abs(out[k, 1] - r[1]) <= REL * max(1.0, abs(r[1]))
