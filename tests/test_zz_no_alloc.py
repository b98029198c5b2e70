"""Allocation-free search entry point (ud_search_device_noalloc), for callers
whose device memory belongs to their own pool allocator or whose loop cannot
take an allocation's device-wide synchronisation: two calls in a row into
caller-owned device buffers give the per-chain results of the ordinary batched
search (ud_search + ud_search_chains) with the same parameters -- at the
default launch shape, at two chains per warp, and on an autotuned batch with
the tuned shape and BFGS cap -- and oversized, malformed or empty requests are
refused before anything launches.

Collected last on purpose: the entry point's scratch is a static device array
whose address is looked up on first use, and this must work both in a fresh
process and after every other test has run kernels on the device."""
import numpy as np
import pytest

from unidock_tools import engine, synth

from .conftest import BOX_CENTER, BOX_SIZE

pytestmark = pytest.mark.gpu

E = 8
MAX_STEP = 10
SEED = 21


@pytest.fixture(scope="module")
def batch(receptor):
    M = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    ligs = [engine.Ligand(synth.make_ligand(12 + 7 * k, k + 1, seed=1300 + k).to_pdbqt()) for k in range(5)]
    B = engine.Batch(M, ligs)
    return M, ligs, B


def _noalloc(B, n_chain, stride, d_evals=True, **shape):
    import torch
    poses = torch.full((n_chain, stride), float("nan"), dtype=torch.float32, device="cuda")
    e = torch.full((n_chain,), float("nan"), dtype=torch.float32, device="cuda")
    ev = torch.full((n_chain,), -1, dtype=torch.int32, device="cuda") if d_evals else None
    stream = torch.cuda.current_stream()
    B.search_device_noalloc(poses.data_ptr(), stride, e.data_ptr(), ev.data_ptr() if d_evals else None,
                            stream.cuda_stream, exhaustiveness=E, max_step=MAX_STEP, seed=SEED, **shape)
    stream.synchronize()
    return poses.cpu().numpy(), e.cpu().numpy(), (ev.cpu().numpy() if d_evals else None)


def _assert_poses_equal(p, ref_p, ligs):
    """Row k holds chain k of ligand k // E; only its first 7 + T floats are
    written (the rest of the row is the caller's)."""
    for k in range(len(ref_p)):
        n = 7 + ligs[k // E].n_torsions
        np.testing.assert_allclose(p[k, :n], ref_p[k, :n], rtol=1e-5, atol=1e-5)


def test_noalloc_matches_batched_search_twice(batch):
    M, ligs, B = batch
    B.search(exhaustiveness=E, max_step=MAX_STEP, seed=SEED, form=1)
    ref_p, ref_e, ref_ev = B.chains()
    n_chain, stride = ref_p.shape
    for _ in range(2):
        p, e, ev = _noalloc(B, n_chain, stride)
        np.testing.assert_allclose(e, ref_e, rtol=1e-5, atol=1e-5)
        np.testing.assert_array_equal(ev, ref_ev)
        _assert_poses_equal(p, ref_p, ligs)
    # a wider caller stride: the columns past each pose are left alone
    import torch
    wide = stride + 3
    poses = torch.zeros((n_chain, wide), dtype=torch.float32, device="cuda")
    e = torch.zeros(n_chain, dtype=torch.float32, device="cuda")
    B.search_device_noalloc(poses.data_ptr(), wide, e.data_ptr(), None, None, exhaustiveness=E,
                            max_step=MAX_STEP, seed=SEED)
    torch.cuda.synchronize()
    got = poses.cpu().numpy()
    _assert_poses_equal(got, ref_p, ligs)
    assert np.all(got[:, stride:] == 0)
    np.testing.assert_allclose(e.cpu().numpy(), ref_e, rtol=1e-5, atol=1e-5)


def test_noalloc_follows_launch_shape_and_tuned_cap(batch):
    """Two chains per warp (another summation order than one chain per warp),
    and an autotuned batch searched with the tuned shape and BFGS cap (0 / 0 /
    -1): the same per-chain results as ud_search with the same parameters."""
    M, ligs, B = batch
    B.search(exhaustiveness=E, max_step=MAX_STEP, seed=SEED, form=1, lanes_per_chain=16, chains_per_block=2)
    ref_p, ref_e, ref_ev = B.chains()
    n_chain, stride = ref_p.shape
    for _ in range(2):
        p, e, ev = _noalloc(B, n_chain, stride, lanes_per_chain=16, chains_per_block=2)
        np.testing.assert_allclose(e, ref_e, rtol=1e-5, atol=1e-5)
        np.testing.assert_array_equal(ev, ref_ev)
        _assert_poses_equal(p, ref_p, ligs)
    T = engine.Batch(M, ligs)
    T.autotune(exhaustiveness=E, max_step=MAX_STEP, seed=SEED)
    T.search(exhaustiveness=E, max_step=MAX_STEP, seed=SEED, form=1, bfgs_cap=-1)
    ref_p, ref_e, ref_ev = T.chains()
    for _ in range(2):
        p, e, ev = _noalloc(T, n_chain, stride, bfgs_cap=-1)
        np.testing.assert_allclose(e, ref_e, rtol=1e-5, atol=1e-5)
        np.testing.assert_array_equal(ev, ref_ev)
        _assert_poses_equal(p, ref_p, ligs)


def test_noalloc_rejects_oversized_and_bad_arguments(batch):
    import torch
    M, ligs, B = batch
    stride = 7 + B.max_torsions
    buf = torch.zeros(64, dtype=torch.float32, device="cuda")
    # 5 ligands x 30000 chains = 150000 > 131072 chains
    with pytest.raises(engine.UdError) as ei:
        B.search_device_noalloc(buf.data_ptr(), stride, buf.data_ptr(), None, None, exhaustiveness=30000)
    assert ei.value.code == engine.UD_ERR_CAPACITY
    assert "131072" in str(ei.value)
    with pytest.raises(engine.UdError) as ei:
        B.search_device_noalloc(buf.data_ptr(), stride - 1, buf.data_ptr(), None, None, exhaustiveness=E)
    assert ei.value.code == engine.UD_ERR_ARG
    with pytest.raises(engine.UdError):
        B.search_device_noalloc(0, stride, buf.data_ptr(), None, None, exhaustiveness=E)
    with pytest.raises(engine.UdError) as ei:
        B.search_device_noalloc(buf.data_ptr(), stride, buf.data_ptr(), None, None, exhaustiveness=E,
                                lanes_per_chain=8)
    assert ei.value.code == engine.UD_ERR_ARG
    # an empty batch is refused, as ud_search refuses it
    empty = engine.Batch(M, [])
    with pytest.raises(engine.UdError) as ei:
        empty.search_device_noalloc(buf.data_ptr(), 7, buf.data_ptr(), None, None, exhaustiveness=E)
    assert ei.value.code == engine.UD_ERR_ARG
    with pytest.raises(engine.UdError) as ei:
        empty.search(exhaustiveness=E)
    assert ei.value.code == engine.UD_ERR_ARG
    torch.cuda.synchronize()
    assert torch.all(buf == 0)
