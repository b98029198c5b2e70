"""Monte-Carlo + BFGS search on the GPU: plain and persistent forms, result
consistency with the fixed-pose energy, and clustering/output."""
import numpy as np
import pytest

from unidock_tools import engine, synth

from .conftest import BOX_CENTER, BOX_SIZE

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(receptor):
    M = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    ligs = [engine.Ligand(synth.make_ligand(14 + 6 * k, k + 1, seed=900 + k).to_pdbqt()) for k in range(4)]
    return M, ligs


@pytest.mark.parametrize("form", [0, 1])
def test_search_chain_energy_is_pose_energy(small, form):
    M, ligs = small
    B = engine.Batch(M, ligs)
    B.search(exhaustiveness=8, max_step=10, seed=3, form=form)
    poses, e, ev = B.chains()
    assert np.all(np.isfinite(e))
    assert np.all(ev > 0)
    lig_of = np.repeat(np.arange(len(ligs)), 8)
    e2, _ = B.score_grad(lig_of, poses, 1000.0, 1000.0)
    np.testing.assert_allclose(e2, e, rtol=1e-4, atol=1e-4)


def test_same_seed_same_result(small):
    M, ligs = small
    B = engine.Batch(M, ligs[:2])
    B.search(exhaustiveness=4, max_step=5, seed=11, form=1)
    _, e1, _ = B.chains()
    B.search(exhaustiveness=4, max_step=5, seed=11, form=0)
    _, e2, _ = B.chains()
    np.testing.assert_allclose(e1, e2, rtol=1e-5)


def test_modes_and_output(small):
    M, ligs = small
    B = engine.Batch(M, ligs)
    B.search(exhaustiveness=16, max_step=10, seed=5, num_modes=9, form=1)
    for li in range(len(ligs)):
        modes = B.modes(li)
        assert 1 <= len(modes) <= 9
        en = np.array([m[1][0] for m in modes])
        assert np.all(np.diff(en) >= 0)
        assert modes[0][1][1] == 0 and modes[0][1][2] == 0   # rmsd to itself
        txt = B.write(li)
        assert txt.startswith("MODEL 1\nREMARK VINA RESULT:")
        assert txt.count("ENDMDL") >= 1
