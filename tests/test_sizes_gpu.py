"""Ligands at the size limits on the GPU, mixed in one batch:
- rigid one-, two- and three-atom ligands (no torsions, no intramolecular pairs);
- the largest the reference parses: 48 torsions, 145 atoms and 7,798
  intramolecular pairs, more than the 4,096 pairs of the reference GPU
  search's largest size bucket (unidock/src/cuda/kernel.h MaxConfig);
- one in between (30 torsions).
Fixed-pose energy and gradient against the reference's FP32 CPU path
(model::eval_deriv, tolerance 1e-4 relative), then a search in both forms,
with refinement, whose chain energies are their poses' energies.  An empty
batch is refused before anything is launched."""
import numpy as np
import pytest

from oracle import ref
from unidock_tools import engine, synth

from .conftest import BOX_CENTER, BOX_SIZE

pytestmark = pytest.mark.gpu

REL = 1e-4
SIZES = [(2, 0, 5), (3, 0, 6), (130, 48, 7), (60, 30, 12), (1, 0, 41)]   # heavy atoms, torsions, seed


@pytest.fixture(scope="module")
def setup(receptor, tmp_path_factory):
    d = tmp_path_factory.mktemp("sizes")
    texts = [synth.make_ligand(nh, nt, seed=s).to_pdbqt() for nh, nt, s in SIZES]
    ligs = [engine.Ligand(t) for t in texts]
    assert [L.n_torsions for L in ligs] == [nt for _, nt, _ in SIZES]
    assert ligs[0].n_pairs == 0 and ligs[2].n_pairs > 4096 and ligs[2].n_atoms <= 150
    paths = []
    for k, t in enumerate(texts):
        p = d / f"l{k}.pdbqt"
        p.write_text(t)
        paths.append(p)
    M = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    return ligs, paths, M


@pytest.mark.skipif(not ref.available(), reason="reference build missing")
@pytest.mark.parametrize("v", [1000.0, 10.0])
def test_energy_and_gradient_match_reference_at_size_limits(setup, receptor, v):
    ligs, paths, M = setup
    R = ref.RefMaps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    B = engine.Batch(M, ligs)
    stride = 7 + B.max_torsions
    for li, (L, p) in enumerate(zip(ligs, paths)):
        RL = ref.RefLigand(p)
        P = synth.random_poses(8, L.n_torsions, -8.0, 8.0, 40 + li)
        full = np.zeros((len(P), stride), np.float32)
        full[:, :P.shape[1]] = P
        e, g = B.score_grad(np.full(len(P), li), full, v, v)
        for k in range(len(P)):
            er, gr, _ = RL.eval_deriv(R, P[k], v, v)
            assert abs(e[k] - er) <= REL * max(1.0, abs(er)), (li, k, e[k], er)
            gk = g[k, :6 + L.n_torsions]
            assert np.linalg.norm(gk - gr) <= REL * max(1.0, np.linalg.norm(gr)), (li, k)


@pytest.mark.parametrize("form", [0, 1])
def test_search_at_size_limits(setup, form):
    ligs, _, M = setup
    E = 8
    B = engine.Batch(M, ligs)
    B.search(exhaustiveness=E, max_step=5, seed=21, form=form, refine_step=3)
    poses, e, ev = B.chains()
    assert np.all(np.isfinite(e)) and np.all(ev > 0)
    e2, _ = B.score_grad(np.repeat(np.arange(len(ligs)), E), poses, 1000.0, 1000.0)
    np.testing.assert_allclose(e2, e, rtol=1e-4, atol=1e-4)
    for li in range(len(ligs)):
        modes = B.modes(li)
        assert 1 <= len(modes) <= 9
        assert np.all(np.isfinite([m[1][0] for m in modes]))
        assert B.write(li).startswith("MODEL 1\nREMARK VINA RESULT:")


def test_empty_batch_is_refused(setup):
    _, _, M = setup
    B = engine.Batch(M, [])
    with pytest.raises(engine.UdError) as e:
        B.search(exhaustiveness=8, max_step=5, seed=1)
    assert e.value.code == engine.UD_ERR_ARG
