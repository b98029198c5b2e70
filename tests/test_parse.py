"""Host parsing/typing/torsion tree against the reference parser
(unidock/src/lib/parse_pdbqt.cpp + model.cpp:initialize) on seeded ligands,
PDBQT and SDF (fragInfo / torsionInfo / atomInfo), and on the reference's own
prepared SDF test inputs when its tree is present."""
import numpy as np
import pytest

from oracle import ref
from unidock_tools import engine, synth

pytestmark = pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) missing")


def assert_same_model(R, M):
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
    np.testing.assert_array_equal(ra["charge"], ma["charge"])


@pytest.mark.parametrize("seed", range(24))
def test_ligand_model_matches_reference(seed, workdir):
    nh = 12 + (seed * 7) % 37
    nt = seed % 11
    lig = synth.make_ligand(nh, nt, seed=100 + seed)
    text = lig.to_pdbqt()
    path = workdir / f"lig{seed}.pdbqt"
    path.write_text(text)
    assert_same_model(ref.RefLigand(path), engine.Ligand(text))


@pytest.mark.parametrize("heavy,torsions,seed", [(1, 0, 41), (2, 0, 5), (3, 0, 6), (60, 30, 12), (130, 48, 7)])
def test_ligand_model_matches_reference_at_size_limits(heavy, torsions, seed, workdir):
    """A one-atom ligand, rigid two- and three-atom ones, and the largest the
    reference parses (48 torsions, 145 atoms): the same model as the
    reference's parser."""
    text = synth.make_ligand(heavy, torsions, seed=seed).to_pdbqt()
    path = workdir / f"limit{heavy}_{torsions}.pdbqt"
    path.write_text(text)
    M = engine.Ligand(text)
    assert M.n_torsions == torsions
    assert_same_model(ref.RefLigand(path), M)


@pytest.mark.parametrize("seed", range(16))
def test_sdf_ligand_model_matches_reference(seed, workdir):
    """SDF front end (parse_sdf_aux / parse_sdf_branch): same atoms in the same
    order, frames, types, charges, tree and pairs as the reference."""
    lig = synth.make_ligand(12 + (seed * 5) % 41, seed % 12, seed=300 + seed, with_charges=True)
    text = lig.to_sdf()
    path = workdir / f"lig{seed}.sdf"
    path.write_text(text)
    M = engine.Ligand(text)
    assert M.torsdof == len(lig.rotatable)
    assert_same_model(ref.RefLigand(path), M)
    # explicit SDF entry point, hydrogens kept: the same model
    assert M.export()["ad"].tolist() == engine.Ligand(text, keep_h=True).export()["ad"].tolist()


@pytest.mark.parametrize("path", ref.reference_inputs("**/*.sdf"), ids=lambda p: p.name)
def test_reference_sdf_inputs_match_reference(path):
    """The reference's own SDF test inputs: prepared ligands (with fragInfo),
    ligands without it (one rigid body) and multi-property records."""
    text = path.read_text()
    try:
        R = ref.RefLigand(path)
    except RuntimeError:
        with pytest.raises(engine.UdError):
            engine.Ligand(text, keep_h=True)
        return
    assert_same_model(R, engine.Ligand(text, keep_h=True))


def test_sdf_without_fragments_is_rigid():
    lig = synth.make_ligand(14, 3, seed=5, with_charges=True)
    text = lig.to_sdf()
    cut = text.index(">  <fragInfo>")
    rigid = text[:cut] + text[text.index(">  <atomInfo>"):]
    M = engine.Ligand(rigid)
    assert (M.n_torsions, M.torsdof) == (0, 0)
    assert M.n_atoms == int(text.split("\n")[3][:3])


def test_sdf_keep_h_false_drops_nonpolar_hydrogens():
    lig = synth.make_ligand(16, 2, seed=9, with_charges=True)
    lines = lig.to_sdf().split("\n")
    # make the last atom a non-polar hydrogen (AutoDock type H) in atomInfo
    k = max(i for i, l in enumerate(lines) if l.rstrip().endswith("HD"))
    lines[k] = lines[k].rstrip()[:-2] + "H "
    text = "\n".join(lines)
    kept, dropped = engine.Ligand(text, keep_h=True), engine.Ligand(text, keep_h=False)
    assert dropped.n_atoms == kept.n_atoms - 1


def test_ligand_write_reproduces_input_record():
    """ud_ligand_write at the input pose: the input lines, with coordinates
    rewritten in their own columns (SDF 1-30, PDBQT 31-54)."""
    lig = synth.make_ligand(22, 4, seed=13, with_charges=True)
    for text, cols in ((lig.to_sdf(), (0, 30)), (lig.to_pdbqt(), (30, 54))):
        M = engine.Ligand(text)
        out = M.write_structure(M.initial_pose())
        src = [l for l in text.split("\n") if "$$$$" not in l]
        dst = out.split("\n")
        assert len(src) == len(dst)
        for a, b in zip(src, dst):
            assert a[:cols[0]] == b[:cols[0]] and a[cols[1]:] == b[cols[1]:]
            if a[cols[0]:cols[1]] != b[cols[0]:cols[1]]:
                w = 10 if cols[0] == 0 else 8
                xa = [float(a[cols[0] + w * k:cols[0] + w * (k + 1)]) for k in range(3)]
                xb = [float(b[cols[0] + w * k:cols[0] + w * (k + 1)]) for k in range(3)]
                np.testing.assert_allclose(xa, xb, atol=1.5e-3)


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


def test_size_limits_refused_at_parse(tmp_path):
    """48 torsions is the largest ligand the reference takes
    (parse_pdbqt.cpp:1107-1113); one more is refused at parse, by both, so a
    screen skips that ligand alone.  Atoms: the engine takes up to 256 (the
    reference 150)."""
    ok = synth.make_ligand(140, 48, seed=7)
    L = engine.Ligand(ok.to_pdbqt())
    assert L.n_torsions == 48 and L.n_atoms <= 256
    over = synth.make_ligand(200, 49, seed=8).to_pdbqt()
    with pytest.raises(engine.UdError) as e:
        engine.Ligand(over)
    assert e.value.code == engine.UD_ERR_CAPACITY and "torsion" in str(e.value)
    big = synth.make_ligand(250, 10, seed=9).to_pdbqt()   # 277 atoms with polar H
    with pytest.raises(engine.UdError) as e:
        engine.Ligand(big)
    assert e.value.code == engine.UD_ERR_CAPACITY and "atom" in str(e.value)
    with pytest.raises(engine.UdError) as e:
        engine.parse_ligands([ok.to_pdbqt(), over, big])
    assert e.value.code == engine.UD_ERR_CAPACITY and "2 of 3" in str(e.value)
    if ref.available():
        p = tmp_path / "over.pdbqt"
        p.write_text(over)
        with pytest.raises(RuntimeError):
            ref.RefLigand(p)
