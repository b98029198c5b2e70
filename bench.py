#!/usr/bin/env python
"""Batched virtual-screen benchmark: ligands/s of the Monte-Carlo + BFGS docking
search on B200, Vina scoring, FP32, search_mode fast (exhaustiveness 128,
max_step 20), synthetic 3,000-atom receptor with a 22.5 A box at 0.375 A
(61^3 points per map) and random-tree ligands (12..48 heavy atoms, 0..10
torsions).  A step is one batch of ligands searched by the batched persistent
form; `value` times the search kernels on device-resident inputs, `e2e` the
whole C-ABI path from PDBQT text to written poses with host buffers.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import contextlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "uni-dock_b200"))

METRIC = "ligands/s on 1 B200, batched vs plain form, at ≤1e-4 rel energy err vs ref"
EXHAUSTIVENESS = 128
MAX_STEP = 20
N_LIGANDS = 4096
BOX = 22.5
SPACING = 0.375
ADJOINT_POSES = 65536
# DRAM bytes (read + write) of one search launch of this workload at 1024
# ligands per step, measured with ncu (dram__bytes_read.sum 18.64 GB +
# dram__bytes_write.sum 0.067 GB, one-pass capture of the first timed launch):
# about 1.3 % of the launch's algorithmic L2 bytes miss L2
SEARCH_LAUNCH_DRAM_BYTES = 18.639e9 + 0.0665e9
# the same for one adjoint launch of the differentiation workload
# (dram__bytes_read.sum 657.0 MB + dram__bytes_write.sum 22.9 MB, ncu --set full)
ADJOINT_LAUNCH_DRAM_BYTES = 657.0e6 + 22.9e6


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=1024, help="ligands per step (per GPU)")
    ap.add_argument("--plain-sample", type=int, default=32, help="ligands timed in the plain form")
    ap.add_argument("--cpu-sample", type=int, default=16, help="ligands timed on the reference CPU path")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--chains-per-block", type=int, default=0, help="warps per CTA (0 = 4)")
    ap.add_argument("--lanes-per-chain", type=int, default=0, choices=[0, 16, 32],
                    help="32 = a warp per chain, 16 = two chains per warp (0 = 32)")
    ap.add_argument("--refine-step", type=int, default=3,
                    help="rounds of refinement against the receptor atoms per mode (0: grid energies only)")
    ap.add_argument("--adjoint-poses", type=int, default=ADJOINT_POSES,
                    help="fixed poses of the adjoint leg (0 = skip)")
    ap.add_argument("--workload", default="screen-fast",
                    choices=["screen-fast", "uneven-vinardo", "uneven-ad4", "stream", "paired"],
                    help="screen-fast: the headline batched screen; the others are the uneven-size detail-mode "
                         "screens (Vinardo, AD4, autotuned), the three-receptor streaming screen and the paired "
                         "one-ligand-one-receptor batches (CLI), each on a sample, printed as their own JSON line")
    ap.add_argument("--stream-ligands", type=int, default=8192, help="ligands per receptor of the streaming screen")
    ap.add_argument("--dry-run", action="store_true",
                    help="no GPU work: every rank builds its ligand shard of the first step and meets the others at "
                         "the timing barrier and max-reduction (gloo), then rank 0 prints a JSON line; checks the "
                         "multi-rank launch on a machine without GPUs")
    ap.add_argument("--profile-case", type=int, default=0,
                    help="profiling aid: search N ligands of the workload twice and exit (no JSON)")
    ap.add_argument("--profile-adjoint", action="store_true",
                    help="profiling aid: the adjoint leg alone (3 warm-up launches and 1 timed, 65,536 poses) "
                         "and exit; the second adjoint launch is the one to capture")
    ap.add_argument("--profile-receptor", type=int, default=3000, choices=[3000, 6000, 12000],
                    help="receptor of the profiling case: 3000 atoms in a 22.5 A box (61^3 maps), "
                         "6000 in 30 A (81^3) or 12000 in 36 A (97^3), as the streaming screen")
    return ap.parse_args()


def profile_case(args):
    """Small case of the same kernel for ncu: the second search launch is the one to capture."""
    import torch
    from unidock_tools import engine, synth
    box = {3000: BOX, 6000: 30.0, 12000: 36.0}[args.profile_receptor]
    rec = synth.make_receptor(args.profile_receptor, seed=1)
    maps = engine.Maps(rec.xyz, rec.xs, np.zeros(3, np.float32), np.full(3, box, np.float32), SPACING)
    ligs = [engine.Ligand(l.to_pdbqt()) for l in
            synth.ligand_set(args.profile_case, seed=20261203, heavy=(12, 48), torsions=(0, 10))]
    b = engine.Batch(maps, ligs)
    P = dict(exhaustiveness=EXHAUSTIVENESS, max_step=MAX_STEP, seed=42, form=1,
             chains_per_block=args.chains_per_block, lanes_per_chain=args.lanes_per_chain,
             refine_step=args.refine_step)
    for _ in range(2):
        b.search_launch(**P)
        torch.cuda.synchronize()
    b.search_collect()
    ev, ms = b.stats()
    dims, _, _, n_maps = maps.info()
    print(f"profile case: {len(ligs)} ligands, receptor {args.profile_receptor} atoms, maps {list(dims)} x {n_maps} "
          f"({int(dims.prod()) * n_maps * 4 / 1e6:.1f} MB), {ev} evals, {ms:.1f} ms", flush=True)


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    def __init__(self):
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self, gpu_index=0):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9 or f[0] != str(gpu_index):
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def flush_l2(torch, buf):
    buf.add_(1.0)  # 256 MB write: larger than the 126 MB L2


# ------------------------------------------------------------------ our arm
def run_ours(args, rank, world):
    import torch
    from unidock_tools import engine, synth

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=180))
    rec = synth.make_receptor(3000, seed=1)
    center = np.zeros(3, np.float32)
    size = np.full(3, BOX, np.float32)
    maps = engine.Maps(rec.xyz, rec.xs, center, size, SPACING)

    steps_total = args.warmup + args.steps
    B = args.batch
    # ligand texts of this rank's batches (weak scaling: every rank searches B
    # ligands per step).  A step's global batch of B * world ligands is split
    # by ligand (unidock_tools.shard, cost-balanced); there is no data-path
    # collective, only the timing barrier and max.
    from unidock_tools.shard import shard
    from unidock_tools.synth import ligand_set
    n_global = max(N_LIGANDS, B * world) if world > 1 else N_LIGANDS
    n_batches = max(1, n_global // (B * world))
    all_ligs = ligand_set(min(n_global, B * world * min(steps_total, n_batches)), seed=20261203,
                          heavy=(12, 48), torsions=(0, 10))
    texts = [l.to_pdbqt() for l in all_ligs]

    def batch_texts(step):
        b = step % n_batches
        glob = texts[b * world * B:(b + 1) * world * B]
        cost = [len(t) for t in glob]  # text length ~ atoms: a cheap cost proxy before parsing
        return [glob[i] for i in shard(len(glob), rank, world, cost)]

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    # refine_step 3: the modes are refined and rescored against the receptor
    # atoms, as the reference's CLI does by default
    P = dict(exhaustiveness=EXHAUSTIVENESS, max_step=MAX_STEP, num_modes=9, min_rmsd=1.0, seed=42, form=1,
             chains_per_block=args.chains_per_block, lanes_per_chain=args.lanes_per_chain, use_graph=1,
             refine_step=args.refine_step)

    # ---- device-resident form: topology uploaded and the search set up (result
    # buffers, ligand order, captured graph) before the timed region
    batches = []
    for s in range(steps_total):
        ligs = engine.parse_ligands(batch_texts(s))
        bt = engine.Batch(maps, ligs)
        bt.search_prepare(**P)
        batches.append((ligs, bt))
    torch.cuda.synchronize()
    for s in range(args.warmup):
        flush_l2(torch, flush)
        batches[s][1].search_launch(**P)
        torch.cuda.synchronize()
        batches[s][1].search_collect()
    clocks = Clocks()
    clocks.start()
    times = []
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    for s in range(args.warmup, steps_total):
        flush_l2(torch, flush)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        batches[s][1].search_launch(**P)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop(dev)
    t_total = sum(times) / 1e3
    if world > 1:
        tt = torch.tensor([t_total], device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t_total = float(tt.item())
    # work accounting of the timed steps (algorithmic bytes and flops per
    # evaluation) and the search kernel's own device time in each of them (CUDA
    # events recorded around the kernel inside the captured graph)
    evals_total, bytes_total, flops_total, kernel_s = 0, 0.0, 0.0, 0.0
    for s in range(args.warmup, steps_total):
        ligs, b = batches[s]
        b.search_collect()
        kernel_s += b.stats()[1] / 1e3
        _, e, ev = b.chains()
        ev = ev.reshape(len(ligs), EXHAUSTIVENESS).sum(axis=1)
        for L, n_ev in zip(ligs, ev):
            ex = L.export()
            n_grid = int(np.sum(ex["xs"] < 36))
            bytes_total += n_ev * (32.0 * n_grid + 16.0 * L.n_pairs)
            flops_total += n_ev * (90.0 * n_grid + 22.0 * L.n_pairs + 50.0 * L.n_nodes)
        evals_total += int(ev.sum())
    ligands_timed = B * args.steps * world
    value = ligands_timed / t_total

    # ---- end-to-end through the public API with host buffers: PDBQT text ->
    # parallel parse -> topology upload -> search (graph: queue reset, kernel,
    # clustering and refinement of the modes, result copies) -> final scores ->
    # output text.  Consecutive
    # batches alternate between two streams, as the CLI runs a screen: the host
    # work of one batch overlaps the search of the next.  Wall-clock time of
    # the whole pipelined loop, device synchronised at both ends.
    # Two batch handles, one per stream, are reused (ud_batch_reset): once they
    # have held the largest batch, nothing is allocated or freed (a device
    # free would wait for the search running on the other stream).
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    h2d = d2h = 0
    pool = []
    for s in range(args.warmup):  # warm the pipeline's code paths and the two handles
        ligs = engine.parse_ligands(batch_texts(s))
        st = streams[s % 2].cuda_stream
        if len(pool) < 2:
            pool.append(engine.Batch(maps, ligs))
        else:
            pool[s % 2].reset(ligs, stream=st)
        bb = pool[s % 2]
        bb.search_launch(**P, stream=st)
        bb.search_collect(stream=st)
        [bb.write(i) for i in range(len(ligs))]
    while len(pool) < 2:
        pool.append(engine.Batch(maps, engine.parse_ligands(batch_texts(0))))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t_e2e0 = time.perf_counter()
    pending = None
    for k, s in enumerate(range(args.warmup, steps_total)):
        st = streams[k % 2].cuda_stream
        ligs = engine.parse_ligands(batch_texts(s))
        bb = pool[k % 2]
        bb.reset(ligs, stream=st)
        # this batch's search starts when the previous batch's graph (search,
        # clustering, refinement) is done: queued behind it on the device, it
        # neither starves that batch's last kernels nor waits for the host
        streams[k % 2].wait_stream(streams[(k + 1) % 2])
        bb.search_launch(**P, stream=st)
        if k == 0:
            n_atoms = sum(L.n_atoms for L in ligs)
            n_nodes = sum(L.n_nodes for L in ligs)
            n_pairs = sum(L.n_pairs for L in ligs)
            h2d = 16 * n_atoms + 40 * n_nodes + 4 * n_pairs + 48 * len(ligs) + 4 * len(ligs)
            stride = 7 + bb.max_torsions
            # chain results, then per ligand the mode count and nine mode slots
            # (chain, pose, refined energies)
            d2h = len(ligs) * EXHAUSTIVENESS * (4 * stride + 24) + len(ligs) * (4 + 9 * (4 + 4 * stride + 16))
        if pending is not None:
            pb, pligs, pst = pending
            pb.search_collect(stream=pst)
            outs = [pb.write(i) for i in range(len(pligs))]
        pending = (bb, ligs, st)
    pb, pligs, pst = pending
    pb.search_collect(stream=pst)
    outs = [pb.write(i) for i in range(len(pligs))]
    torch.cuda.synchronize()
    e2e_t = time.perf_counter() - t_e2e0
    del pending, pb, pligs, bb, ligs, pool
    if world > 1:
        tt = torch.tensor([e2e_t], device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        e2e_t = float(tt.item())
    e2e_value = ligands_timed / e2e_t

    # ---- plain form: one launch per ligand with fixed tiling, same search parameters
    plain = None
    if rank == 0 and args.plain_sample > 0:
        ligs, b = batches[args.warmup]
        sub = ligs[:args.plain_sample]
        bp = engine.Batch(maps, sub)
        bp.search_launch(**dict(P, form=0, use_graph=0))
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        bp.search_launch(**dict(P, form=0, use_graph=0))
        e1.record()
        torch.cuda.synchronize()
        bp.search_collect()
        plain = len(sub) / (e0.elapsed_time(e1) / 1e3)

    adjoint = adjoint_leg(maps, engine.l2_peak_gbs()) if rank == 0 and args.adjoint_poses > 0 else None

    result = None
    if rank == 0:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        fp32_peak = engine.fp32_peak_tflops()
        l2_peak = engine.l2_peak_gbs()
        ms_launch = kernel_s * 1e3 / args.steps
        achieved_gbs = bytes_total / kernel_s / 1e9
        achieved_tf = flops_total / kernel_s / 1e12
        result = {
            "metric": METRIC, "value": round(value, 3), "unit": "ligands/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_total * 1e3 / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded receptor, random-tree ligands)",
            "config": {"workload": "batched virtual screen, Vina, search_mode fast (exhaustiveness 128, "
                                   "max_step 20), 4096 ligands U{12..48} heavy / U{0..10} torsions, "
                                   "3000-atom receptor, 22.5 A box at 0.375 A (61^3)",
                       "ligands_per_step": B * world, "exhaustiveness": EXHAUSTIVENESS, "max_step": MAX_STEP,
                       "refine_step": args.refine_step,
                       "warps_per_cta": args.chains_per_block or 4, "lanes_per_chain": args.lanes_per_chain or 32,
                       "form": "batched persistent", "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"ligand shards x{world}" if world > 1 else "1 GPU"},
            "plain_form_ligands_per_s": None if plain is None else round(plain, 3),
            "batched_over_plain": None if plain is None else round(value / plain, 2),
            "evals_per_s": round(evals_total / t_total, 1),
            # the search reads L2-resident maps and pair tables: its memory
            # ceiling is L2 read bandwidth (measured here), not HBM; about
            # 1.3 % of its L2 reads go on to DRAM
            "roofline": {"bound": "l2", "achieved": round(achieved_gbs, 2), "peak": round(l2_peak, 1),
                         "unit": "GB/s", "frac": round(achieved_gbs / l2_peak, 4),
                         "traffic": SEARCH_LAUNCH_DRAM_BYTES if B == 1024 else None,
                         "traffic_note": "DRAM bytes (read + write) per launch from one ncu capture of this "
                                         "workload; the achieved figure counts algorithmic L2 bytes per "
                                         "evaluation (32 per grid atom + 16 per intramolecular pair)",
                         "peak_source": "measured L2 read probe on this GPU (ud_device_l2_peak: 32 MB buffer, "
                                        "16-byte L2-only loads from every SM, best of 5, CUDA events)",
                         "kernel": "ud::dev::search_kernel",
                         "ms_per_launch": round(ms_launch, 3),
                         "timing": "CUDA events recorded around the search kernel inside each timed step's graph",
                         "hbm": {"achieved": round(SEARCH_LAUNCH_DRAM_BYTES / (ms_launch / 1e3) / 1e9, 2)
                                 if B == 1024 else None, "peak": hbm_peak, "unit": "GB/s",
                                 "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)"},
                         "fp32": {"achieved": round(achieved_tf, 3), "peak": round(fp32_peak, 2),
                                  "unit": "TFLOP/s", "frac": round(achieved_tf / fp32_peak, 4),
                                  "peak_source": "measured FMA probe (ud_device_fp32_peak)"}},
            "e2e": {"value": round(e2e_value, 3), "unit": "ligands/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "path": "PDBQT text -> parse (all host threads) -> upload into a reused batch handle -> "
                            "graph (search kernel, clustering and refinement of the modes on the device, result "
                            "copies) -> final scores -> output text; batches pipelined on two streams, wall clock"},
            "clocks": clk,
            # per step: the search kernel, the clustering kernel and (refine_step > 0) the refinement kernel
            "gpu_launches": args.steps * (3 if args.refine_step > 0 else 2),
            "adjoint": adjoint,
        }
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return result


def adjoint_leg(maps, l2_peak, n_ligands=256, reps=5):
    """Differentiation workload: 65,536 fixed poses over 256 ligands of the
    screen's size distribution (centre uniform in the box, uniform random unit
    quaternion, torsions U(-pi, pi)); energy + pose-layout gradient + the 6
    term-weight gradients per pose in one adjoint launch (exact pair
    derivative).  Device-resident inputs, CUDA-event time of the launch."""
    import torch
    from unidock_tools import engine, synth
    ligs = [engine.Ligand(l.to_pdbqt()) for l in
            synth.ligand_set(n_ligands, seed=7, heavy=(12, 48), torsions=(0, 10))]
    B = engine.Batch(maps, ligs)
    per = ADJOINT_POSES // n_ligands
    stride = 7 + B.max_torsions
    P = np.zeros((n_ligands * per, stride), np.float32)
    for i, L in enumerate(ligs):
        P[i * per:(i + 1) * per, :7 + L.n_torsions] = synth.random_poses(per, L.n_torsions, -BOX / 2, BOX / 2,
                                                                          seed=1000 + i)
    n = len(P)
    nt = maps.n_terms
    d_p = torch.from_numpy(P).cuda()
    d_l = torch.from_numpy(np.repeat(np.arange(n_ligands, dtype=np.int32), per)).cuda()
    d_e = torch.empty(n, device="cuda")
    d_g = torch.empty((n, stride), device="cuda")
    d_w = torch.empty((n, nt), device="cuda")
    s = torch.cuda.current_stream().cuda_stream

    def run():
        B.score_adjoint_device(d_l.data_ptr(), d_p.data_ptr(), n, stride, d_e.data_ptr(), d_g.data_ptr(), stride,
                               d_w.data_ptr(), nt, exact=True, stream=s)
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    # algorithmic bytes per launch: per pose the weighted maps and pair rows
    # once for the energy / pose gradient and once per term for the weight
    # gradient (32 B per grid atom and map set, 16 B per pair and table), plus
    # the pose in and the energy, gradient and weight gradient out
    per_lig = []
    for L in ligs:
        n_grid = int(np.sum(L.export()["xs"] < 36))
        per_lig.append((1 + nt) * (32.0 * n_grid + 16.0 * L.n_pairs) + 4.0 * (stride + 1 + stride + nt))
    bytes_launch = per * float(np.sum(per_lig))
    gbs = bytes_launch / (ms / 1e3) / 1e9
    return {"workload": f"{n} fixed poses over {n_ligands} ligands, Vina, energy + pose gradient + "
                        f"{nt} term-weight gradients (exact), FP32", "poses_per_s": round(n / (ms / 1e3), 1),
            "ms_per_launch": round(ms, 3),
            "roofline": {"bound": "l2", "kernel": "ud::dev::adjoint_kernel", "achieved": round(gbs, 1),
                         "peak": round(l2_peak, 1), "unit": "GB/s", "frac": round(gbs / l2_peak, 4),
                         "algorithmic_bytes_per_launch": round(bytes_launch),
                         "traffic": ADJOINT_LAUNCH_DRAM_BYTES if n == ADJOINT_POSES and n_ligands == 256 else None,
                         "traffic_note": "DRAM bytes (read + write) per launch from one ncu capture of this workload",
                         "note": "the 7 map sets (weighted + 6 term maps, 153 MB at 61^3) exceed the 126 MB L2, "
                                 "so part of the reads come from HBM"}}


# ------------------------------------------------------------------ other workloads
def run_uneven(args, sf_name):
    """Uneven-size screen: lognormal heavy-atom counts (median 28, 8..80), torsions
    min(n/4, Poisson(6)) <= 20, search_mode detail (exhaustiveness 512, max_step 40),
    Vinardo or AD4 (receptor and ligand charges N(0, 0.25 e), integer net charge),
    chains-per-CTA and BFGS cap picked by the autotuner on each batch."""
    import torch
    from unidock_tools import engine, synth
    per_step = args.batch if args.batch != 1024 else 512
    rec = synth.make_receptor(3000, seed=1, with_charges=(sf_name == "ad4"))
    center, size = np.zeros(3, np.float32), np.full(3, BOX, np.float32)
    if sf_name == "ad4":
        xyz, xs, ad, q = engine.parse_receptor_ex(rec.to_pdbqt())
        maps = engine.Maps(xyz, ad, center, size, SPACING, sf=engine.SF_AD4, charges=q)
    else:
        maps = engine.Maps(rec.xyz, rec.xs, center, size, SPACING, sf=engine.SF_VINARDO)
    steps_total = args.warmup + args.steps
    texts = [l.to_pdbqt() for l in synth.ligand_set(per_step * steps_total, seed=8192, dist="lognormal",
                                                      with_charges=(sf_name == "ad4"))]
    P = dict(exhaustiveness=512, max_step=40, seed=42, form=1, use_graph=1, chains_per_block=0, bfgs_cap=-1,
             lanes_per_chain=0, refine_step=args.refine_step)
    batches, tunes = [], []
    for s in range(steps_total):
        ligs = engine.parse_ligands(texts[s * per_step:(s + 1) * per_step])
        bt = engine.Batch(maps, ligs)
        tunes.append(bt.autotune(exhaustiveness=512, max_step=40, seed=42))
        bt.search_prepare(**P)
        batches.append(bt)
    for s in range(args.warmup):
        batches[s].search_launch(**P)
        torch.cuda.synchronize()
    times, evals = [], 0
    for s in range(args.warmup, steps_total):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        batches[s].search_launch(**P)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
        batches[s].search_collect()
        evals += batches[s].stats()[0]
    t = sum(times)
    tune = tunes[args.warmup]
    return {"metric": "ligands/s on 1 B200 (uneven-size screen)", "value": round(per_step * args.steps / t, 3),
            "unit": "ligands/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * t / args.steps, 1), "higher_is_better": True, "dtype": "f32",
            "data": "synthetic", "evals_per_s": round(evals / t, 1),
            "config": {"workload": f"uneven-size screen, {sf_name}, search_mode detail (exhaustiveness 512, "
                                   "max_step 40), lognormal sizes (median 28 heavy, 8..80), 3000-atom receptor, "
                                   "22.5 A box", "ligands_per_step": per_step,
                       "autotuned": {k: tune[k] for k in ("chains_per_block", "lanes_per_chain", "bfgs_cap",
                                                          "energy_shift",
                                                          "ligands_per_s", "base_ligands_per_s")}}}


def run_paired(args):
    """Paired 1:1 batches through the CLI (--paired_batch_size): 64 complexes,
    each its own synthetic receptor (8 receptors of 3000 atoms, boxes
    centred on their pockets) and ligand, search_mode fast settings, batches
    of 16; wall clock of the whole command, files in and out."""
    import json
    import subprocess
    import tempfile
    from unidock_tools import synth
    n_rec, n_cplx, batch = 8, 64, 16
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        cfg = {}
        for r in range(n_rec):
            (d / f"rec{r}.pdbqt").write_text(synth.make_receptor(3000, seed=500 + r).to_pdbqt())
        ligs = synth.ligand_set(n_cplx, seed=777, heavy=(12, 48), torsions=(0, 10))
        for k, L in enumerate(ligs):
            (d / f"lig{k}.pdbqt").write_text(L.to_pdbqt())
            (d / f"lig{k}_config.json").write_text(json.dumps(
                {"center_x": 0.0, "center_y": 0.0, "center_z": 0.0, "size_x": BOX, "size_y": BOX, "size_z": BOX}))
            cfg[f"c{k}"] = {"protein": str(d / f"rec{k % n_rec}.pdbqt"), "ligand": str(d / f"lig{k}.pdbqt"),
                            "ligand_config": str(d / f"lig{k}_config.json")}
        (d / "pairs.json").write_text(json.dumps(cfg))
        (d / "out").mkdir()
        cmd = [str(ROOT / "uni-dock_b200" / "bin" / "unidock"), "--paired_batch_size", str(batch), "--ligand_index",
               str(d / "pairs.json"), "--dir", str(d / "out"), "--size_x", str(BOX), "--size_y", str(BOX),
               "--size_z", str(BOX), "--exhaustiveness", str(EXHAUSTIVENESS), "--max_step", str(MAX_STEP),
               "--seed", "5"]
        t0 = time.perf_counter()
        r = subprocess.run(cmd, capture_output=True, text=True)
        t = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(r.stdout + r.stderr)
        done = len(list((d / "out").glob("*_out.pdbqt")))
    return {"metric": "complexes/s (paired one-ligand-one-receptor batches)", "value": round(done / t, 3),
            "unit": "complexes/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded receptors and random-tree ligands)",
            "config": {"workload": f"paired batches: {n_cplx} complexes over {n_rec} receptors (3000 atoms each), "
                                   f"box {BOX} A at {SPACING} A, exhaustiveness {EXHAUSTIVENESS}, max_step "
                                   f"{MAX_STEP}, refine_step 3, --paired_batch_size {batch}",
                       "timing": "wall clock of the CLI command: receptor parsing, map builds (complexes of a "
                                 "batch with the same receptor and box share one), searches queued on 16 streams, "
                                 "refinement, output files"},
            "complexes_done": done, "seconds": round(t, 3)}


def run_stream(args):
    """Streaming screen: search_mode balance (exhaustiveness 384, max_step 40),
    ligands with U{10..100} heavy atoms and U{0..30} torsions, fed slot by slot
    (64 ligands a slot, 4 result areas) into one persistent search kernel per
    receptor (ud_stream_*), against three receptors: 3000 atoms with a 22.5 A
    box, 6000 with 30 A, 12000 with 36 A (0.375 A).  The host parses each slot,
    pushes it while the kernel works on earlier ones, and collects (clustering,
    refinement, final scores) and writes each finished slot's results; the
    wall clock from the first push to the kernel's end gives sustained
    ligands/s."""
    import torch
    from unidock_tools import engine, synth
    n_lig = args.stream_ligands
    slot, ring = 64, 4
    n_slots = (n_lig + slot - 1) // slot
    out = []
    for n_rec, box in ((3000, 22.5), (6000, 30.0), (12000, 36.0)):
        rec = synth.make_receptor(n_rec, seed=1)
        maps = engine.Maps(rec.xyz, rec.xs, np.zeros(3, np.float32), np.full(3, box, np.float32), SPACING)
        dims, _, _, n_maps = maps.info()
        texts = [l.to_pdbqt() for l in synth.ligand_set(n_lig, seed=100000 + n_rec, heavy=(10, 100),
                                                        torsions=(0, 30))]
        # the stream's per-chain shared memory is sized for the largest ligand it takes
        probe = engine.parse_ligands(texts)
        max_atoms = max(L.n_atoms for L in probe)
        max_tors = max(L.n_torsions for L in probe)
        del probe
        torch.cuda.synchronize()
        st = engine.Stream(maps, exhaustiveness=384, max_step=40, seed=42, refine_step=args.refine_step,
                           slot_ligands=slot, max_slots=n_slots, ring=ring, max_atoms=max_atoms,
                           max_torsions=max_tors, timeout_ms=120000)
        t0 = time.perf_counter()
        held = {}
        written = 0
        for k in range(n_slots):
            ligs = engine.parse_ligands(texts[k * slot:(k + 1) * slot])
            if k >= ring:  # the result area of slot k - ring is reused by slot k
                st.collect(k - ring)
                written += sum(len(st.write(k - ring, i)) > 0 for i in range(len(held[k - ring])))
                del held[k - ring]
            st.push(ligs)
            held[k] = ligs
        st.close()
        for k in sorted(held):
            st.collect(k)
            written += sum(len(st.write(k, i)) > 0 for i in range(len(held[k])))
        evals = st.finish()
        t = time.perf_counter() - t0
        del st
        map_bytes = int(dims.prod()) * n_maps * 4
        out.append({"receptor_atoms": n_rec, "box": box, "grid": [int(d) for d in dims], "ligands": n_lig,
                    "ligands_written": int(written), "ligands_per_s": round(n_lig / t, 2),
                    "evals_per_s": round(evals / t, 1), "seconds": round(t, 1),
                    "max_atoms": int(max_atoms), "max_torsions": int(max_tors),
                    "map_mbytes": round(map_bytes / 1e6, 1), "xpair_map_mbytes": round(2 * map_bytes / 1e6, 1),
                    "maps_fit_l2_126mb": map_bytes < 126e6})
    return {"metric": "sustained ligands/s on 1 B200 (streaming screen)", "unit": "ligands/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "value": round(min(r["ligands_per_s"] for r in out), 3),
            "config": {"workload": "streaming screen, Vina, search_mode balance (exhaustiveness 384, max_step 40), "
                                   "ligands U{10..100} heavy / U{0..30} torsions, one persistent kernel per "
                                   "receptor fed 64-ligand slots from page-locked memory (4 result areas), "
                                   f"refine_step {args.refine_step}, wall clock from the first push to the "
                                   "kernel's end", "ligands_per_slot": slot, "receptors": out}}


# ------------------------------------------------------------------ reference CPU path
@contextlib.contextmanager
def c_stdout_to_stderr():
    """The reference's own code prints diagnostics with printf; while it runs,
    file descriptor 1 points at stderr so that stdout carries the JSON line
    alone."""
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        os.dup2(saved, 1)
        os.close(saved)


def reference_cpu(sample, step_index, threads=None, seed=7):
    with c_stdout_to_stderr():
        return _reference_cpu(sample, step_index, threads, seed)


def _reference_cpu(sample, step_index, threads=None, seed=7):
    """The reference's CPU docking at the screen's settings on `sample` ligands
    of the same generator, all the reference's own code (oracle/_ref, built
    from its sources): its parallel Monte-Carlo search (parallel_mc over
    monte_carlo::operator(), the machinery of Vina::global_search,
    vina.cpp:1495-1540) with the step count capped at max_step as its GPU path
    caps it, then the refinement of every mode against the receptor atoms and
    the final scores (vina.h:232-343), on all host threads.  The maps are built
    once outside the timing, as a screen builds them once per receptor.
    Returns ligands/s and the threads used."""
    sys.path.insert(0, str(ROOT))
    from oracle import ref
    from unidock_tools import synth
    if not ref.gpu_available():
        raise RuntimeError("oracle/_ref/libudref_gpu.so missing (build it with make -C oracle)")
    threads = threads or os.cpu_count()
    rec = synth.make_receptor(3000, seed=1)
    maps = ref.RefMaps(rec.xyz, rec.xs, np.zeros(3, np.float32), np.full(3, BOX, np.float32), SPACING)
    ligs = synth.ligand_set(sample * (step_index + 1), seed=20261203, heavy=(12, 48), torsions=(0, 10))
    ligs = ligs[sample * step_index:]
    maxf = float(np.finfo(np.float32).max)
    t_total = 0.0
    with tempfile.TemporaryDirectory() as d:
        for k, L in enumerate(ligs):
            p = Path(d) / f"l{k}.pdbqt"
            p.write_text(L.to_pdbqt())
            R = ref.RefLigand(p)
            t0 = time.perf_counter()
            _, poses = ref.parallel_mc(R, maps, EXHAUSTIVENESS, MAX_STEP, seed + k, threads)
            refined, order_e = [], []
            for pose in poses:
                rp, e_last, _, _, within = R.refine(maps, pose, 3)
                refined.append(rp)
                order_e.append(e_last if within else maxf)
            R.final_scores(maps, np.array(refined, np.float32), order_e, receptor=True)
            t_total += time.perf_counter() - t0
    return len(ligs) / t_total, threads


SINGLE_DOCKING = "plain single docking: Vina, 3000-atom receptor, 22.5 A box at 0.375 A, one ligand of 24 " \
    "heavy atoms and 6 torsions, exhaustiveness 8, num_modes 9, heuristic step count, refinement 3 steps"


def single_docking_files(d):
    from unidock_tools import synth
    rp, lp = Path(d) / "rec.pdbqt", Path(d) / "lig.pdbqt"
    rp.write_text(synth.make_receptor(3000, seed=1).to_pdbqt())
    lp.write_text(synth.make_ligand(24, 6, seed=31).to_pdbqt())
    return rp, lp


def single_docking_reference(threads=None):
    with c_stdout_to_stderr():
        return _single_docking_reference(threads)


def _single_docking_reference(threads=None):
    """The plain single docking through the reference's stock CPU docking of one ligand
    (Vina::set_receptor .. global_search, the reference CLI's --cpu path):
    wall clock of the whole call and the best mode's energy."""
    sys.path.insert(0, str(ROOT))
    from oracle import ref
    threads = threads or os.cpu_count()
    with tempfile.TemporaryDirectory() as d:
        rp, lp = single_docking_files(d)
        t0 = time.perf_counter()
        e = ref.vina_dock(rp, lp, np.zeros(3), np.full(3, BOX), SPACING, 8, 9, 5, threads)
        t = time.perf_counter() - t0
    return {"workload": SINGLE_DOCKING, "path": "reference CPU Vina::global_search (stock CPU path, whole call)",
            "seconds": round(t, 3), "cores": threads, "best_energy": round(float(e[0]), 3)}


def single_docking_engine():
    """The plain single docking through this engine's C ABI, one ligand: receptor parse, map
    build, ligand parse, search (exhaustiveness 8, the heuristic step count),
    clustering, refinement and final scores, output text; wall clock."""
    import torch
    from unidock_tools import engine
    with tempfile.TemporaryDirectory() as d:
        rp, lp = single_docking_files(d)
        for rep in range(2):  # the first call pays module loading and allocation
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            xyz, xs = engine.parse_receptor(rp.read_text())
            maps = engine.Maps(xyz, xs, np.zeros(3, np.float32), np.full(3, BOX, np.float32), SPACING)
            L = engine.Ligand(lp.read_text())
            B = engine.Batch(maps, [L])
            B.search(exhaustiveness=8, max_step=0, num_modes=9, seed=5, refine_step=3)
            text = B.write(0)
            torch.cuda.synchronize()
            t = time.perf_counter() - t0
    return {"workload": SINGLE_DOCKING, "path": "this engine's C ABI: parse, maps, search, clustering, refinement, output",
            "seconds": round(t, 3), "best_energy": round(float(B.modes(0)[0][1][0]), 3),
            "output_bytes": len(text)}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    sample = max(1, args.cpu_sample)
    for s in range(args.warmup):
        reference_cpu(1, s)
    vals = []
    for s in range(args.steps):
        v, thr = reference_cpu(sample, args.warmup + s)
        vals.append(v)
    value = len(vals) * sample / sum(sample / v for v in vals)
    try:
        c0 = single_docking_reference()
    except Exception as ex:  # the single-docking leg never blocks the line
        c0 = {"workload": SINGLE_DOCKING, "unavailable": str(ex)}
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "ligands/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sample / value, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded receptor, random-tree ligands)",
        "config": {"workload": "batched virtual screen, Vina, search_mode fast (exhaustiveness 128, max_step 20), "
                               "4096 ligands U{12..48} heavy / U{0..10} torsions, 3000-atom receptor, 22.5 A box",
                   "sample_ligands_per_step": sample},
        "cpu_baseline": {"value": round(value, 4), "unit": "ligands/s", "cores": thr, "kind": "reference",
                         "sample": f"{sample} ligands per step x {args.steps} steps: the reference's parallel_mc "
                                   "(128 tasks of monte_carlo::operator(), 20 MC steps each) then refinement and "
                                   "final scores of every mode, the reference's own sources built by oracle/Makefile"},
        "e2e": {"value": round(value, 4), "unit": "ligands/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "single_docking": c0,
    }


def relaunch(args) -> int:
    """`--gpus N` (N > 1) run directly: start N ranks of this script under
    torch.distributed.run on this node (rendezvous on 127.0.0.1) and return
    their exit status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve())] + sys.argv[1:]
    return subprocess.call(cmd)


def run_dry(args, rank, world):
    """The multi-rank plumbing without a GPU: each rank's ligand shard of the
    first step, the timing barrier and the max over ranks (gloo)."""
    import torch
    import torch.distributed as dist
    from unidock_tools.shard import shard
    from unidock_tools.synth import ligand_set
    if world > 1:
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    B = args.batch
    texts = [l.to_pdbqt() for l in ligand_set(B * world, seed=20261203, heavy=(12, 48), torsions=(0, 10))]
    mine = shard(len(texts), rank, world, [len(t) for t in texts])
    t = torch.tensor([float(len(mine))])
    n = torch.tensor([float(len(mine))])
    if world > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
        dist.destroy_process_group()
    if rank != 0:
        return None
    return {"dry_run": True, "metric": METRIC, "n_gpus": world, "ligands_per_step": B * world,
            "ligands_sharded": int(n.item()), "max_rank_ligands": int(t.item()), "scaling": "weak"}


def main():
    args = parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch(args))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        raise SystemExit(f"bench.py --gpus {args.gpus} launched with WORLD_SIZE={world}: one rank per GPU expected")
    if args.dry_run:
        res = run_dry(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    if args.profile_case > 0:
        profile_case(args)
        return
    if args.profile_adjoint:
        from unidock_tools import engine, synth
        rec = synth.make_receptor(3000, seed=1)
        maps = engine.Maps(rec.xyz, rec.xs, np.zeros(3, np.float32), np.full(3, BOX, np.float32), SPACING)
        print(json.dumps(adjoint_leg(maps, engine.l2_peak_gbs(), reps=1)), flush=True)
        return
    if args.workload != "screen-fast" and args.impl != "reference":
        res = (run_stream(args) if args.workload == "stream" else
               run_paired(args) if args.workload == "paired" else run_uneven(args, args.workload.split("-")[1]))
        print(json.dumps(res), flush=True)
        return
    if args.impl == "reference":
        res = run_reference(args, rank, world)
    else:
        res = run_ours(args, rank, world)
        if res is not None and world == 1 and not args.no_cpu_baseline:
            try:
                v, thr = reference_cpu(args.cpu_sample, 0)
                res["cpu_baseline"] = {"value": round(v, 4), "unit": "ligands/s", "cores": thr, "kind": "reference",
                                       "sample": f"{args.cpu_sample} ligands: the reference's parallel_mc (128 "
                                                 "tasks, 20 MC steps each), refinement and final scores of every "
                                                 "mode, on all host threads"}
            except Exception as ex:  # the baseline never blocks the GPU line
                res["cpu_baseline"] = {"value": None, "unit": "ligands/s", "cores": os.cpu_count(),
                                       "kind": "reference", "sample": f"unavailable: {ex}"}
    if res is not None and args.impl != "reference" and world == 1 and not args.no_cpu_baseline:
        try:
            res["single_docking"] = {"engine": single_docking_engine(), "reference": single_docking_reference()}
        except Exception as ex:
            res["single_docking"] = {"workload": SINGLE_DOCKING, "unavailable": str(ex)}
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
