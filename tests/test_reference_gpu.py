"""The reference's own GPU batched search (unidock/src/cuda/monte_carlo.cu
kernel + precalculate.cu tables, built for sm_100a by oracle/Makefile) against
the engine on the same GPU, the same ligands and the same search settings
(search_mode fast: exhaustiveness 128, max_step 20).

The reference groups ligands into size buckets and runs one launch per bucket
(unidock/src/main/main.cpp:95-118, 1040-1070); so does this test.  Its time is
the reference's do_docking (host marshalling, kernel, result conversion) plus
its per-ligand pair tables; the engine's is one search launch with the modes
clustered on the device.  Both sides' best energies are reported: the two
searches draw different random streams, so they are compared as
distributions."""
import time

import numpy as np
import pytest

from oracle import ref
from unidock_tools import engine, synth

from .conftest import BOX_CENTER, BOX_SIZE

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.gpu_available(), reason="reference GPU build missing")]

N_LIGANDS = 256
E, MAX_STEP = 128, 20


def test_engine_beats_reference_gpu_kernel(receptor, tmp_path, capfd):
    import re
    import torch
    ligs = synth.ligand_set(N_LIGANDS, seed=20261203, heavy=(12, 48), torsions=(0, 10))
    refs, ours = [], []
    for k, L in enumerate(ligs):
        p = tmp_path / f"l{k}.pdbqt"
        p.write_text(L.to_pdbqt())
        refs.append(ref.RefLigand(p))
        ours.append(engine.Ligand(L.to_pdbqt()))
    R = ref.RefMaps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    buckets = {}
    for i, RL in enumerate(refs):
        b = ref.gpu_bucket(RL)
        assert b >= 0
        buckets.setdefault(b, []).append(i)
    ref_best = np.full(N_LIGANDS, np.nan, np.float32)
    t_ref = 0.0
    for b, idx in sorted(buckets.items()):
        best, t_tables, t_dock, cfg = ref.gpu_dock(R, [refs[i] for i in idx], E, MAX_STEP, 42)
        assert cfg == b
        ref_best[idx] = best
        t_ref += t_tables + t_dock
    assert np.all(np.isfinite(ref_best))
    # the reference times its own kernel launches (monte_carlo.cu: "Time spend on GPU is ... ms")
    t_ref_kernel = sum(float(x) for x in re.findall(r"Time spend on GPU is ([0-9.]+) ms", capfd.readouterr().out)) / 1e3

    M = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375)
    B = engine.Batch(M, ours)
    P = dict(exhaustiveness=E, max_step=MAX_STEP, seed=42, use_graph=1)
    B.search(**P)  # warm: buffers, graph
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    B.search(**P)
    t_ours = time.perf_counter() - t0
    _, kernel_ms = B.stats()
    _, ce, _ = B.chains()
    our_chain_best = ce.reshape(N_LIGANDS, E).min(axis=1)

    with capfd.disabled():
        report(N_LIGANDS, buckets, t_ref, t_ref_kernel, t_ours, kernel_ms, ref_best, our_chain_best)
    assert t_ours < t_ref
    assert kernel_ms / 1e3 < t_ref_kernel


def report(n, buckets, t_ref, t_ref_kernel, t_ours, kernel_ms, ref_best, our_chain_best):
    print(f"\nreference GPU search: {n / t_ref:.2f} ligands/s ({t_ref:.2f} s with its pair tables; "
          f"buckets {dict(sorted((b, len(i)) for b, i in buckets.items()))}), its kernels alone "
          f"{n / t_ref_kernel:.2f} ligands/s ({t_ref_kernel:.3f} s)")
    print(f"engine: {n / t_ours:.2f} ligands/s ({t_ours:.3f} s for ud_search), its graph alone "
          f"{n / (kernel_ms / 1e3):.2f} ligands/s ({kernel_ms / 1e3:.3f} s); speed-up {t_ref / t_ours:.1f}x "
          f"end to end, {t_ref_kernel / (kernel_ms / 1e3):.1f}x kernels")
    # like with like: both numbers are the search's own energy (the best over
    # a ligand's chains of the refined pose energy, inter + intra at curl cap
    # 1000), before clustering, refinement and the final conf-independent score
    print(f"median chain-best search energy: reference GPU kernel {np.median(ref_best):.3f}, engine "
          f"{np.median(our_chain_best):.3f} kcal/mol")
