"""Streaming screen (ud_stream_*): one persistent search kernel fed slot by
slot from page-locked host memory while it runs.

  * two rings' worth of slots (ring 2, 4 slots of 16 ligands; each slot
    pushed only after the slot two before it was collected) give exactly the
    per-chain results of one batched search (ud_search) of the same 64
    ligands with the same seed: a ligand's global id in the stream (slot x 16
    + position) is its index in the batch, and so are its random streams;
  * with refinement, the modes and final scores of every ligand equal the
    batched search's;
  * the host stops feeding (no close): the kernel's wait for the next slot
    runs out after its 1 s limit and ud_stream_finish reports UD_ERR_TIMEOUT,
    with the context still usable;
  * malformed requests are refused before anything is copied.
"""
import time

import numpy as np
import pytest

from unidock_tools import engine, synth

from .conftest import BOX_CENTER, BOX_SIZE

pytestmark = pytest.mark.gpu

E = 8
MAX_STEP = 10
SEED = 31
SLOT = 16
SLOTS = 4


@pytest.fixture(scope="module")
def setup(receptor):
    maps = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    texts = [l.to_pdbqt() for l in synth.ligand_set(SLOT * SLOTS, seed=515, heavy=(12, 40), torsions=(0, 8))]
    ligs = [engine.Ligand(t) for t in texts]
    max_atoms = max(L.n_atoms for L in ligs)
    max_tors = max(L.n_torsions for L in ligs)
    return maps, ligs, max_atoms, max_tors


def stream_all(maps, ligs, max_atoms, max_tors, refine_step=0, ring=2):
    st = engine.Stream(maps, exhaustiveness=E, max_step=MAX_STEP, seed=SEED, refine_step=refine_step,
                       slot_ligands=SLOT, max_slots=SLOTS, ring=ring, max_atoms=max_atoms,
                       max_torsions=max_tors, timeout_ms=20000)
    out = {}
    for k in range(SLOTS):
        if k >= ring:  # the result area of slot k - ring is reused by slot k
            st.collect(k - ring)
            out[k - ring] = (st.chains(k - ring), [st.modes(k - ring, i) for i in range(SLOT)])
        assert st.push(ligs[k * SLOT:(k + 1) * SLOT]) == k
    st.close()
    for k in range(max(0, SLOTS - ring), SLOTS):
        st.collect(k)
        out[k] = (st.chains(k), [st.modes(k, i) for i in range(SLOT)])
    evals = st.finish()
    return out, evals


def test_stream_equals_batched_chains(setup):
    maps, ligs, max_atoms, max_tors = setup
    out, evals = stream_all(maps, ligs, max_atoms, max_tors)
    B = engine.Batch(maps, ligs)
    B.search(exhaustiveness=E, max_step=MAX_STEP, seed=SEED, form=1, lanes_per_chain=32)
    bp, be, bev = B.chains()
    assert evals == int(bev.sum())
    for k in range(SLOTS):
        (p, e, ev), _ = out[k]
        rows = slice(k * SLOT * E, (k + 1) * SLOT * E)
        np.testing.assert_array_equal(ev, bev[rows])
        np.testing.assert_allclose(e, be[rows], rtol=1e-6, atol=1e-6)
        for i in range(SLOT * E):
            T = ligs[k * SLOT + i // E].n_torsions
            np.testing.assert_allclose(p[i, :7 + T], bp[rows][i, :7 + T], rtol=1e-6, atol=1e-6)
    print(f"stream of {SLOTS} slots x {SLOT} ligands (ring 2): {evals} evaluations, chains equal to the batched search")


def test_stream_modes_equal_batched_modes(setup):
    maps, ligs, max_atoms, max_tors = setup
    out, _ = stream_all(maps, ligs, max_atoms, max_tors, refine_step=3)
    B = engine.Batch(maps, ligs)
    B.search(exhaustiveness=E, max_step=MAX_STEP, seed=SEED, form=1, lanes_per_chain=32, refine_step=3)
    for k in range(SLOTS):
        _, modes = out[k]
        for i in range(SLOT):
            ref = B.modes(k * SLOT + i)
            assert len(modes[i]) == len(ref)
            for (pa, ea), (pb, eb) in zip(modes[i], ref):
                np.testing.assert_allclose(pa, pb, rtol=1e-5, atol=1e-5)
                np.testing.assert_allclose(ea, eb, rtol=1e-5, atol=1e-5)


def test_stream_wait_times_out_when_the_host_stops_feeding(setup):
    maps, ligs, max_atoms, max_tors = setup
    st = engine.Stream(maps, exhaustiveness=E, max_step=MAX_STEP, seed=SEED, slot_ligands=SLOT, max_slots=SLOTS,
                       ring=2, max_atoms=max_atoms, max_torsions=max_tors, timeout_ms=1000)
    st.push(ligs[:SLOT])
    st.collect(0)  # the published slot is done; nothing further is published and the stream is not closed
    t0 = time.perf_counter()
    with pytest.raises(engine.UdError) as ei:
        st.finish()
    waited = time.perf_counter() - t0
    assert ei.value.code == engine.UD_ERR_TIMEOUT
    assert waited < 30
    _, e, _ = st.chains(0)
    assert np.all(np.isfinite(e))
    # the context is still usable
    B = engine.Batch(maps, ligs[:2])
    B.search(exhaustiveness=2, max_step=2, seed=1)
    print(f"kernel gave up waiting {waited:.2f} s after the last slot was collected")


def test_stream_refuses_bad_requests(setup):
    maps, ligs, max_atoms, max_tors = setup
    with pytest.raises(engine.UdError) as ei:
        engine.Stream(maps, exhaustiveness=E, max_step=0, slot_ligands=SLOT, max_atoms=max_atoms,
                      max_torsions=max_tors)
    assert ei.value.code == engine.UD_ERR_ARG
    st = engine.Stream(maps, exhaustiveness=E, max_step=MAX_STEP, seed=SEED, slot_ligands=SLOT, max_slots=3,
                       ring=1, max_atoms=max_atoms, max_torsions=max_tors, timeout_ms=20000)
    big = engine.Ligand(synth.make_ligand(max_atoms, 2, seed=99).to_pdbqt())
    if big.n_atoms > max_atoms:
        with pytest.raises(engine.UdError) as ei:
            st.push([big])
        assert ei.value.code == engine.UD_ERR_CAPACITY
    with pytest.raises(engine.UdError) as ei:
        st.push(ligs[:SLOT + 1])  # more than a slot holds
    assert ei.value.code == engine.UD_ERR_ARG
    st.push(ligs[:4])
    with pytest.raises(engine.UdError) as ei:
        st.push(ligs[4:8])  # ring 1: slot 0 must be collected first
    assert ei.value.code == engine.UD_ERR_STATE
    st.collect(0)
    st.push(ligs[4:8])
    st.close()
    st.collect(1)
    st.finish()
