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


@pytest.mark.parametrize("form,lanes", [(0, 32), (1, 32), (1, 16)])
def test_search_chain_energy_is_pose_energy(small, form, lanes):
    M, ligs = small
    B = engine.Batch(M, ligs)
    B.search(exhaustiveness=8, max_step=10, seed=3, form=form, lanes_per_chain=lanes)
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


def test_vinardo_search_chain_energy_is_pose_energy(receptor):
    M = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375, sf=engine.SF_VINARDO)
    ligs = [engine.Ligand(synth.make_ligand(16 + 8 * k, 2 * k + 1, seed=1700 + k).to_pdbqt()) for k in range(3)]
    B = engine.Batch(M, ligs)
    B.search(exhaustiveness=8, max_step=10, seed=4, form=1)
    poses, e, ev = B.chains()
    assert np.all(np.isfinite(e)) and np.all(ev > 0)
    e2, _ = B.score_grad(np.repeat(np.arange(len(ligs)), 8), poses, 1000.0, 1000.0)
    np.testing.assert_allclose(e2, e, rtol=1e-4, atol=1e-4)
    for li in range(len(ligs)):
        assert B.write(li).startswith("MODEL 1\nREMARK VINA RESULT:")


def test_graph_form_equals_persistent_form(small):
    M, ligs = small
    B = engine.Batch(M, ligs)
    B.search(exhaustiveness=8, max_step=8, seed=13, form=1, use_graph=0)
    p0, e0, ev0 = B.chains()
    for _ in range(2):  # captured once, replayed
        B.search(exhaustiveness=8, max_step=8, seed=13, form=1, use_graph=1)
        p1, e1, ev1 = B.chains()
        np.testing.assert_array_equal(e1, e0)
        np.testing.assert_array_equal(ev1, ev0)
    B.search(exhaustiveness=8, max_step=8, seed=14, form=1, use_graph=1)   # new parameters: recaptured
    _, e2, _ = B.chains()
    B.search(exhaustiveness=8, max_step=8, seed=14, form=1, use_graph=0)
    _, e3, _ = B.chains()
    np.testing.assert_array_equal(e2, e3)
    assert B.write(0).startswith("MODEL 1\nREMARK VINA RESULT:")


def test_autotune_picks_valid_configuration(small):
    M, ligs = small
    B = engine.Batch(M, ligs * 8)
    r = B.autotune(exhaustiveness=16, max_step=6, seed=1)
    assert r["chains_per_block"] in (1, 2, 4)
    assert r["bfgs_cap"] == 0  # BFGS caps are not tuned
    assert r["lanes_per_chain"] in (16, 32) and r["n_tried"] == 6
    assert r["energy_shift"] <= 0.1 and r["ligands_per_s"] >= r["base_ligands_per_s"] > 0
    B.search(exhaustiveness=16, max_step=6, seed=1, form=1, chains_per_block=0, bfgs_cap=-1)
    _, e, ev = B.chains()
    assert np.all(np.isfinite(e)) and np.all(ev > 0)


@pytest.mark.parametrize("warps", [1, 2, 4])
def test_half_warp_chains(small, warps):
    """Two chains per warp (16 lanes each): deterministic for a seed, the
    captured graph replays the direct launch exactly, chain energies are their
    poses' energies, and every chain's random stream is its own, so the
    results track the one-chain-per-warp search (same streams, a different
    FP32 summation order, so the trajectories part after a few steps): over
    64 chains per ligand the median chain energies of the two widths differ
    by at most 0.3 kcal/mol beyond twice the bootstrap standard error of the
    difference."""
    M, ligs = small
    B = engine.Batch(M, ligs)
    P = dict(exhaustiveness=8, max_step=8, seed=13, form=1, chains_per_block=warps, lanes_per_chain=16)
    B.search(use_graph=0, **P)
    p0, e0, ev0 = B.chains()
    B.search(use_graph=1, **P)
    p1, e1, ev1 = B.chains()
    np.testing.assert_array_equal(e1, e0)
    np.testing.assert_array_equal(ev1, ev0)
    e2, _ = B.score_grad(np.repeat(np.arange(len(ligs)), 8), p0, 1000.0, 1000.0)
    np.testing.assert_allclose(e2, e0, rtol=1e-4, atol=1e-4)
    Pt = dict(P, exhaustiveness=64, use_graph=0)
    B.search(**Pt)
    _, e16, _ = B.chains()
    B.search(**dict(Pt, lanes_per_chain=32))
    _, e32, _ = B.chains()
    rng = np.random.default_rng(5)
    d = float(np.median(e16) - np.median(e32))
    se = float(np.std([np.median(rng.choice(e16, len(e16))) - np.median(rng.choice(e32, len(e32)))
                       for _ in range(1000)]))
    print(f"{warps} warps per CTA: median chain energy 16 lanes {np.median(e16):.3f}, 32 lanes {np.median(e32):.3f} "
          f"(diff {d:+.3f}, se {se:.3f})")
    assert abs(d) <= 0.3 + 2 * se
    with pytest.raises(engine.UdError):
        B.search(**dict(P, lanes_per_chain=8))


def test_prepare_then_launch_equals_search(small):
    M, ligs = small
    B = engine.Batch(M, ligs)
    B.search_prepare(exhaustiveness=8, max_step=6, seed=21, form=1, use_graph=1)
    B.search_launch(exhaustiveness=8, max_step=6, seed=21, form=1, use_graph=1)
    B.search_collect()
    _, e1, ev1 = B.chains()
    B2 = engine.Batch(M, ligs)
    B2.search(exhaustiveness=8, max_step=6, seed=21, form=1, use_graph=0)
    _, e2, ev2 = B2.chains()
    np.testing.assert_array_equal(e1, e2)
    np.testing.assert_array_equal(ev1, ev2)
    assert [m[1][0] for m in B.modes(0)] == [m[1][0] for m in B2.modes(0)]


def test_reset_batch_equals_fresh_batch(small):
    """A batch handle reused for other ligands (ud_batch_reset) searches
    exactly as a fresh batch of them: a smaller batch, a larger one, and one
    with the same ligand count, largest ligand and step count but more atoms in
    total (topology arrays reallocated under an otherwise unchanged graph)."""
    M, ligs = small
    B = engine.Batch(M, [ligs[3], ligs[0]])
    P = dict(exhaustiveness=8, max_step=6, seed=21, use_graph=1, refine_step=3)
    B.search(**P)
    for sub in ([ligs[3], ligs[2]], ligs[:1], ligs):
        B.reset(sub)
        B.search(**P)
        F = engine.Batch(M, sub)
        F.search(**P)
        _, e_reset, _ = B.chains()
        _, e_fresh, _ = F.chains()
        np.testing.assert_array_equal(e_reset, e_fresh)
        for li in range(len(sub)):
            a, b = B.modes(li), F.modes(li)
            assert len(a) == len(b)
            for (pa, ea), (pb, eb) in zip(a, b):
                np.testing.assert_array_equal(pa, pb)
                np.testing.assert_array_equal(ea, eb)
