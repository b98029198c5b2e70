"""Bias wells (AutoDock-bias style BPF, --bias / --multi_bias) against the
reference's own code: the wells added to the maps (cache::compute_bias) within
1e-5 of the map's scale, and energies and gradients against the receptor
atoms with the maps' wells or a ligand's own wells (non_cache with bias,
model::bias_list): energies within 1e-4, gradients within 2e-4 (summation
order over the receptor atoms; see the test).  AutoDock 4.2 maps: the wells
of ad4cache::set_bias within 1e-5 of each map's scale."""
import numpy as np
import pytest

from oracle import ref
from unidock_tools import engine, synth

from .conftest import BOX_CENTER, BOX_SIZE

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference build missing")]

# acceptor wells, map wells for named AD types (one naming two carbon types,
# which the receptor-atom scoring counts twice), a donor and an aromatic well
# (no effect in XS scoring) and an unknown type
BPF = """x y z Vset r type
 2.0  1.0 -1.5 -2.0 1.2 acc
-3.0  0.5  2.0 -1.5 1.5 map C A N
 0.5 -2.5  0.0 -3.0 1.0 map OA
 1.0  1.0  1.0 -2.0 1.0 don
-1.0  2.0 -2.0 -2.0 1.0 aro
 0.0  0.0  4.0 -1.0 2.0 what
"""
LIG_BPF = """x y z Vset r type
-2.0 -1.0  1.0 -2.5 1.3 map C
 1.5  2.5 -0.5 -2.0 1.1 acc
"""


@pytest.fixture(scope="module")
def setup(receptor, tmp_path_factory):
    d = tmp_path_factory.mktemp("bias")
    ligs, refs = [], []
    for k in range(4):
        L = synth.make_ligand(16 + 6 * k, 2 * k + 1, seed=1300 + k)
        p = d / f"l{k}.pdbqt"
        p.write_text(L.to_pdbqt())
        ligs.append(engine.Ligand(L.to_pdbqt()))
        refs.append(ref.RefLigand(p))
    M = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    M.add_bias(BPF)
    R = ref.RefMaps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    assert R.add_bias(BPF) == 6
    return ligs, refs, M, R


def test_bias_maps_match_reference(setup):
    ligs, refs, M, R = setup
    changed = 0
    for xs in range(36):
        want = R.get(xs)
        if want is None:
            continue
        try:
            got = M.read(xs)
        except engine.UdError:
            continue
        scale = max(1.0, float(np.abs(want).max()))
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-5 * scale, err_msg=f"XS type {xs}")
        changed += 1
    assert changed >= 10


@pytest.mark.parametrize("own", [False, True])
def test_bias_receptor_energies_match_reference(setup, own):
    ligs, refs, M, R = setup
    B = engine.Batch(M, ligs)
    if own:
        for li, RL in enumerate(refs):
            B.set_bias(li, LIG_BPF)
            RL.set_bias(LIG_BPF)
    stride = 7 + B.max_torsions
    for li, (L, RL) in enumerate(zip(ligs, refs)):
        P = synth.random_poses(10, L.n_torsions, -5.0, 5.0, seed=li + 71)
        full = np.zeros((len(P), stride), np.float32)
        full[:, :P.shape[1]] = P
        e, g = B.score_grad_receptor(np.full(len(P), li), full, 1e6, 1000.0)
        for k in range(len(P)):
            er, gr = RL.nc_eval_deriv(R, P[k], 1e6, 1000.0)
            assert abs(e[k] - er) <= 1e-4 * max(1.0, abs(er)), (li, k, e[k], er)
            gk = g[k, :6 + L.n_torsions]
            # 2e-4: both sides sum ~190 receptor atoms per ligand atom in FP32, the
            # reference in sequence, the GPU over lanes; at close contacts the
            # cancelling pair forces leave ~1e-4 of the gradient's norm to
            # summation order, with or without wells (the wells' own share of the
            # gradient agrees to 4e-6)
            assert np.linalg.norm(gk - gr) <= 2e-4 * max(1.0, np.linalg.norm(gr)), (li, k)
    if own:
        for RL in refs:
            RL.set_bias("x y z Vset r type\n")


def test_bias_changes_the_maps_and_blocks_term_weights(setup, receptor):
    ligs, refs, M, R = setup
    plain = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    assert np.abs(M.read(8) - plain.read(8)).max() > 0.01  # O_A: acceptor and OA map wells
    with pytest.raises(engine.UdError):
        M.set_weights(M.weights())


# AutoDock 4.2 maps: donor wells go to HD, acceptor wells to OA and NA,
# aromatic wells to A, map wells to the AD types named or, with none named,
# to every map including the electrostatic and desolvation maps
AD4_BPF = """x y z Vset r type
 1.0  2.0 -1.5 -2.0 1.2 don
-3.0  0.5  2.0 -1.5 1.0 acc
 2.5 -2.0  1.0 -1.0 1.5 aro
 0.0  0.0  0.0 -0.8 2.0 map C OA
-1.0  3.0 -2.0 -0.6 1.1 map
 0.0  0.0  4.0 -1.0 2.0 what
"""


def test_ad4_bias_maps_match_reference(tmp_path):
    """--bias with --scoring ad4: the engine's AD4 maps are written as AutoGrid
    files and read by the reference's ad4cache; both then add the same wells
    (ad4cache::set_bias, ad4cache.cpp:54-88, against ud_maps_add_bias), and
    every map, the electrostatic and desolvation maps included, agrees within
    1e-5 of its scale, and every map changed (the untyped map well reaches
    them all).  A search on the biased maps then runs."""
    rec = synth.make_receptor(3000, seed=1, with_charges=True)
    xyz, _, ad, q = engine.parse_receptor_ex(rec.to_pdbqt())
    M = engine.Maps(xyz, ad, BOX_CENTER, BOX_SIZE, 0.375, sf=engine.SF_AD4, charges=q)
    prefix = str(tmp_path / "rec")
    M.write(prefix)
    R = ref.RefAd4Maps(prefix)
    dims = M.info()[0]
    n = int(dims.prod())
    before = {}
    for t in range(37):
        try:
            before[t] = M.read(t).ravel().copy()
        except engine.UdError:
            pass
    assert R.add_bias(AD4_BPF) == 6
    M.add_bias(AD4_BPF)
    changed, compared = set(), 0
    for t, b in before.items():
        got = M.read(t).ravel()
        want = R.get(t, n)
        assert want is not None, t
        scale = max(1.0, float(np.abs(want).max()))
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-5 * scale, err_msg=f"AD4 map {t}")
        compared += 1
        if np.any(got != b):
            changed.add(t)
    AD_A, AD_C, AD_NA, AD_OA, AD_HD = 1, 0, 9, 10, 12
    # the all-maps well reaches every map; the typed wells add to their own
    assert changed == set(before), (sorted(changed), sorted(before))
    for t in (AD_A, AD_C, AD_NA, AD_OA, AD_HD, 35, 36):
        if t in before:
            assert t in changed
    print(f"AD4 bias: {compared} maps compared with the reference, {len(changed)} changed")
    # a search on the biased maps runs
    lig = engine.Ligand(synth.ligand_set(1, seed=4242, dist="lognormal", with_charges=True)[0].to_pdbqt())
    B = engine.Batch(M, [lig])
    B.search(exhaustiveness=8, max_step=5, seed=3)
    assert B.modes(0)
