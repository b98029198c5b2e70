"""SDF ligands on the GPU: fixed-pose energies and gradients of SDF-parsed
models against the reference's FP32 CPU path on the same SDF files (its
parse_sdf_ligand model), the same molecule read from SDF and from PDBQT
scoring alike, and search results written back as SDF records
(model::write_sdf_model, unidock/src/lib/model.cpp:850-866)."""
import numpy as np
import pytest

from oracle import ref
from unidock_tools import engine, synth

from .conftest import BOX_CENTER, BOX_SIZE

pytestmark = pytest.mark.gpu

REL = 1e-4


@pytest.fixture(scope="module")
def setup(receptor, tmp_path_factory):
    d = tmp_path_factory.mktemp("sdf")
    mols = [synth.make_ligand(14 + 6 * k, min(2 * k, 10), seed=700 + k, with_charges=True) for k in range(6)]
    for L in mols:  # PDBQT keeps 3 decimals, SDF 4: give both files the same coordinates
        L.heavy_xyz = np.round(L.heavy_xyz, 3)
        L.h_xyz = [(a, np.round(h, 3)) for a, h in L.h_xyz]
    paths, sdf, pdbqt = [], [], []
    for k, L in enumerate(mols):
        p = d / f"l{k}.sdf"
        p.write_text(L.to_sdf())
        paths.append(p)
        sdf.append(engine.Ligand(L.to_sdf()))
        pdbqt.append(engine.Ligand(L.to_pdbqt()))
    M = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    return mols, paths, sdf, pdbqt, M


@pytest.mark.skipif(not ref.available(), reason="reference build missing")
def test_sdf_model_energy_and_gradient_match_reference(setup, receptor):
    mols, paths, sdf, _, M = setup
    R = ref.RefMaps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    B = engine.Batch(M, sdf)
    stride = 7 + B.max_torsions
    for li, (L, p) in enumerate(zip(sdf, paths)):
        RL = ref.RefLigand(p)
        P = synth.random_poses(12, L.n_torsions, -8.0, 8.0, seed=40 + li)
        full = np.zeros((len(P), stride), np.float32)
        full[:, :P.shape[1]] = P
        e, g = B.score_grad(np.full(len(P), li), full)
        for k in range(len(P)):
            er, gr, _ = RL.eval_deriv(R, P[k])
            assert abs(e[k] - er) <= REL * max(1.0, abs(er)), (li, k, e[k], er)
            gk = g[k, :6 + L.n_torsions]
            assert np.linalg.norm(gk - gr) <= REL * max(1.0, np.linalg.norm(gr)), (li, k)


def test_sdf_and_pdbqt_of_one_molecule_score_alike(setup):
    """Atom order and torsion tree differ between the two files of one
    molecule; the energy at the input coordinates does not (up to FP32
    summation order)."""
    _, _, sdf, pdbqt, M = setup
    for a, b in zip(sdf, pdbqt):
        assert (a.n_atoms, a.n_torsions, a.n_pairs) == (b.n_atoms, b.n_torsions, b.n_pairs)
        ea, _ = engine.Batch(M, [a]).score_grad(np.zeros(1, np.int32), a.initial_pose()[None, :])
        eb, _ = engine.Batch(M, [b]).score_grad(np.zeros(1, np.int32), b.initial_pose()[None, :])
        assert abs(ea[0] - eb[0]) <= 1e-4 * max(1.0, abs(eb[0])), (ea, eb)


def test_search_results_written_as_sdf_records(setup):
    mols, _, sdf, _, M = setup
    B = engine.Batch(M, sdf)
    B.search(exhaustiveness=8, max_step=10, num_modes=4, seed=181129)
    for li, L in enumerate(mols):
        src = [l for l in L.to_sdf().split("\n") if l and "$$$$" not in l]
        text = B.write(li, 1)
        records = text.split("$$$$\n")
        assert records[-1] == ""
        records = records[:-1]
        assert 1 <= len(records) <= 4
        energies = []
        for r in records:
            head, result = r.split("> <Uni-Dock RESULT> \n")
            lines = [l for l in head.split("\n") if l]
            assert len(lines) == len(src)
            moved = 0
            for a, b in zip(src, lines):
                # atom lines: new x/y/z in columns 1-30, the rest of the line unchanged
                assert a[30:] == b[30:]
                moved += a[:30] != b[:30]
            assert moved > 0
            assert result.startswith("ENERGY=")
            energies.append(float(result.split("\n")[0][len("ENERGY="):].split()[0]))
            assert "INTER + INTRA:" in result and "UNBOUND:" in result
        assert energies == sorted(energies)
        assert all(np.isfinite(energies))
