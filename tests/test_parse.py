"""Host parsing/typing/torsion tree against the reference parser
(unidock/src/lib/parse_pdbqt.cpp + model.cpp:initialize) on seeded ligands."""
import numpy as np
import pytest

from oracle import ref
from unidock_tools import engine, synth

pytestmark = pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) missing")


@pytest.mark.parametrize("seed", range(24))
def test_ligand_model_matches_reference(seed, workdir):
    nh = 12 + (seed * 7) % 37
    nt = seed % 11
    lig = synth.make_ligand(nh, nt, seed=100 + seed)
    text = lig.to_pdbqt()
    path = workdir / f"lig{seed}.pdbqt"
    path.write_text(text)
    R = ref.RefLigand(path)
    M = engine.Ligand(text)
    ra, ma = R.atoms(), M.export()
    assert (R.n_atoms, R.n_torsions, R.n_pairs) == (M.n_atoms, M.n_torsions, M.n_pairs)
    for k in ("xs", "ad", "el"):
        np.testing.assert_array_equal(ra[k], ma[k])
    np.testing.assert_array_equal(ra["local"], ma["local"])
    np.testing.assert_array_equal(ra["lab"], ma["lab"])
    pa, pb = R.pairs()
    np.testing.assert_array_equal(pa, ma["pair_a"])
    np.testing.assert_array_equal(pb, ma["pair_b"])
    par, beg, end, rel = R.tree()
    np.testing.assert_array_equal(par, ma["parent"])
    np.testing.assert_array_equal(beg, ma["begin"])
    np.testing.assert_array_equal(end, ma["end"])
    np.testing.assert_array_equal(rel, ma["rel"])
    np.testing.assert_array_equal(R.conf_indep()[:6], M.conf_indep()[:6])


def test_initial_pose_reproduces_input_coordinates():
    lig = synth.make_ligand(30, 6, seed=7)
    M = engine.Ligand(lig.to_pdbqt())
    xyz = M.coords(M.initial_pose())
    np.testing.assert_allclose(xyz, M.export()["lab"], atol=2e-5)


def test_malformed_inputs_raise():
    with pytest.raises(engine.UdError):
        engine.Ligand("ROOT\nENDROOT\nTORSDOF 0\n")          # no atoms
    good = synth.make_ligand(12, 2, seed=3).to_pdbqt()
    with pytest.raises(engine.UdError):
        engine.Ligand(good.replace("TORSDOF", "REMARK"))      # missing TORSDOF
    with pytest.raises(engine.UdError):
        engine.Ligand(good.replace("ENDBRANCH", "ENDBRANCH 99", 1))
