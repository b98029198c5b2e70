"""The unidock command-line host: the reference's option surface and argument
checks (no GPU needed), and on the GPU a batch docking run that writes one
`<ligand>_out.pdbqt` per input ligand in --dir, a single-ligand run with the
default output name, and --score_only / --local_only."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from unidock_tools import synth

ROOT = Path(__file__).resolve().parent.parent
BIN = ROOT / "uni-dock_b200" / "bin" / "unidock"

# option names of the reference CLI (unidock/src/main/main.cpp:421-575)
REFERENCE_OPTIONS = [
    "receptor", "flex", "ligand", "ligand_index", "paired_batch_size", "batch", "gpu_batch", "scoring", "maps",
    "center_x", "center_y", "center_z", "size_x", "size_y", "size_z", "autobox", "out", "dir", "write_maps",
    "device_id", "score_only", "score_file", "local_only", "no_refine", "force_even_voxels", "randomize_only",
    "weight_gauss1", "weight_gauss2", "weight_repulsion", "weight_hydrophobic", "weight_hydrogen", "weight_rot",
    "weight_vinardo_gauss1", "weight_vinardo_repulsion", "weight_vinardo_hydrophobic", "weight_vinardo_hydrogen",
    "weight_vinardo_rot", "weight_ad4_vdw", "weight_ad4_hb", "weight_ad4_elec", "weight_ad4_dsolv",
    "weight_ad4_rot", "weight_glue", "bias", "multi_bias", "keep_nonpolar_H", "cpu", "seed", "exhaustiveness",
    "max_evals", "num_modes", "min_rmsd", "energy_range", "spacing", "verbosity", "max_step", "refine_step",
    "max_gpu_memory", "search_mode", "config", "help", "help_advanced", "version"]


def run(*args, cwd=None):
    return subprocess.run([str(BIN), *map(str, args)], capture_output=True, text=True, cwd=cwd, timeout=600)


def test_help_lists_every_reference_option():
    r = run("--help_advanced")
    assert r.returncode == 0
    for name in REFERENCE_OPTIONS:
        assert f"--{name} " in r.stdout, name


@pytest.mark.parametrize("args,msg", [
    (["--receptor", "r.pdbqt"], "Missing ligand(s)."),
    (["--receptor", "r.pdbqt", "--gpu_batch", "a.pdbqt"], "Need to specify an output directory for batch mode."),
    (["--receptor", "r.pdbqt", "--gpu_batch", "a.pdbqt", "--dir", "/nonexistent_dir_x"], "does not exist"),
    (["--receptor", "r.pdbqt", "--ligand", "a.pdbqt", "--scoring", "xyz"], "Scoring function xyz unknown."),
    (["--receptor", "r.pdbqt", "--ligand", "a.pdbqt", "--flex", "f.pdbqt"], "--flex is not supported by this engine"),
    (["--ligand", "a.pdbqt"], "The receptor or affinity maps must be specified."),
    (["--bogus", "1"], "unrecognised option '--bogus'"),
    (["--receptor", "r.pdbqt", "--ligand", "a.pdbqt", "--gpu_batch", "b.pdbqt", "--dir", "."],
     "Can't use both --ligand and --batch arguments simultaneously."),
    (["--receptor", "r.pdbqt", "--ligand", "a.pdbqt", "--search_mode", "slow"], "unknown search_mode"),
    (["--paired_batch_size", "2"], "ERROR: Paired batch size set, but no config json specified via --ligand_index"),
    (["--paired_batch_size", "2", "--ligand_index", "c.json"], "ERROR: Need to specify an output directory for batch mode."),
])
def test_argument_errors(args, msg):
    r = run(*args)
    assert r.returncode != 0
    assert msg in r.stderr + r.stdout, (r.stdout, r.stderr)


def box_args(size=22.5):
    return ["--center_x", 0, "--center_y", 0, "--center_z", 0, "--size_x", size, "--size_y", size, "--size_z", size]


@pytest.fixture(scope="module")
def inputs(tmp_path_factory, receptor):
    d = tmp_path_factory.mktemp("cli")
    (d / "rec.pdbqt").write_text(receptor.to_pdbqt())
    names = []
    for k, L in enumerate(synth.ligand_set(6, seed=77, heavy=(12, 30), torsions=(0, 6))):
        p = d / f"lig{k}.pdbqt"
        p.write_text(L.to_pdbqt())
        names.append(p)
    (d / "out").mkdir()
    return d, names


@pytest.mark.gpu
def test_batch_docking_writes_one_output_per_ligand(inputs):
    d, names = inputs
    idx = d / "index.txt"
    idx.write_text("\n".join(str(p) for p in names[3:]) + "\n")
    r = run("--receptor", d / "rec.pdbqt", "--gpu_batch", *names[:3], "--ligand_index", idx, "--dir", d / "out",
            "--search_mode", "fast", "--seed", 3, "--num_modes", 5, "--batch_size", 4, *box_args())
    assert r.returncode == 0, r.stderr
    assert "Batch 1 size: 4" in r.stdout and "Batch 2 size: 2" in r.stdout
    for p in names:
        out = d / "out" / (p.stem + "_out.pdbqt")
        text = out.read_text()
        assert text.startswith("MODEL 1\nREMARK VINA RESULT:")
        assert 1 <= text.count("ENDMDL") <= 5
        e = [float(l.split()[3]) for l in text.splitlines() if l.startswith("REMARK VINA RESULT:")]
        assert e == sorted(e) and e[-1] <= e[0] + 3.0 + 1e-6


@pytest.mark.gpu
def test_oversized_ligand_is_skipped_alone(inputs, tmp_path):
    """A ligand over the torsion limit is reported and skipped; the rest of the
    screen is docked (parse_ligand_from_file_no_failure, parse_pdbqt.cpp:1107-1113)."""
    d, names = inputs
    big = tmp_path / "big.pdbqt"
    big.write_text(synth.make_ligand(200, 49, seed=8).to_pdbqt())
    out = tmp_path / "out"
    out.mkdir()
    r = run("--receptor", d / "rec.pdbqt", "--gpu_batch", names[0], big, names[1], "--dir", out,
            "--exhaustiveness", 8, "--max_step", 5, "--seed", 2, *box_args())
    assert r.returncode == 0, r.stderr
    assert "skipping ligand" in r.stderr and "exceeds max torsion counts" in r.stderr
    assert not (out / "big_out.pdbqt").exists()
    for p in names[:2]:
        assert (out / (p.stem + "_out.pdbqt")).read_text().startswith("MODEL 1\nREMARK VINA RESULT:")


@pytest.mark.gpu
def test_max_gpu_memory_packs_smaller_batches(inputs, tmp_path):
    """--max_gpu_memory caps the device memory of the batches in flight: a
    budget of about a megabyte per batch splits six ligands over several
    batches and still docks every one; a budget below the maps' own memory is
    refused."""
    import re
    d, names = inputs
    common = ["--receptor", d / "rec.pdbqt", "--gpu_batch", *names, "--exhaustiveness", 2048, "--max_step", 1,
              "--seed", 4, *box_args()]
    out1 = tmp_path / "o1"
    out1.mkdir()
    r = run(*common, "--dir", out1, "--verbosity", 2)
    assert r.returncode == 0, r.stderr
    used = int(re.search(r"GPU memory: maps (\d+) MiB", r.stdout).group(1))
    assert "Batch 2 size" not in r.stdout
    out2 = tmp_path / "o2"
    out2.mkdir()
    r = run(*common, "--dir", out2, "--max_gpu_memory", used + 66)   # 64 MiB reserve + about 1 MiB per batch
    assert r.returncode == 0, r.stderr
    sizes = [int(x) for x in re.findall(r"Batch \d+ size: (\d+)", r.stdout)]
    assert len(sizes) >= 2 and sum(sizes) == len(names)
    for p in names:
        assert (out2 / (p.stem + "_out.pdbqt")).read_text().startswith("MODEL 1\nREMARK VINA RESULT:")
    r = run(*common, "--dir", out2, "--max_gpu_memory", 1)
    assert r.returncode != 0 and "max_gpu_memory" in r.stderr


@pytest.mark.gpu
def test_single_ligand_default_output_and_modes_table(inputs):
    d, names = inputs
    r = run("--receptor", d / "rec.pdbqt", "--ligand", names[0], "--exhaustiveness", 8, "--max_step", 10,
            "--seed", 1, *box_args())
    assert r.returncode == 0, r.stderr
    assert "mode |   affinity | dist from best mode" in r.stdout
    out = names[0].with_name(names[0].stem + "_out.pdbqt")
    assert out.read_text().startswith("MODEL 1\nREMARK VINA RESULT:")


@pytest.mark.gpu
def test_score_only_and_local_only(inputs):
    d, names = inputs
    r = run("--receptor", d / "rec.pdbqt", "--ligand", names[1], "--score_only", *box_args())
    assert r.returncode == 0, r.stderr
    assert "Estimated Free Energy of Binding" in r.stdout
    score = names[1].with_name(names[1].stem + "_score.txt").read_text()
    assert score.startswith(f"REMARK {names[1].name} ")
    assert np.isfinite(float(score.split()[2]))
    out = d / "local.pdbqt"
    r = run("--receptor", d / "rec.pdbqt", "--ligand", names[1], "--local_only", "--out", out, *box_args())
    assert r.returncode == 0, r.stderr
    # the input structure with new coordinates, line for line
    src, dst = names[1].read_text().splitlines(), out.read_text().splitlines()
    assert len(src) == len(dst)
    moved = 0
    for a, b in zip(src, dst):
        if a.startswith(("ATOM", "HETATM")):
            assert a[:30] == b[:30] and a[54:] == b[54:]
            moved += a[30:54] != b[30:54]
        else:
            assert a == b
    assert moved > 0
    r = run("--receptor", d / "rec.pdbqt", "--ligand", names[1], "--score_only", "--autobox")
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("scoring", ["vina", "vinardo"])
def test_sdf_batch_docking(inputs, tmp_path, scoring):
    """SDF ligands through --gpu_batch (the reference's test_unidock_sdf.py
    case: --search_mode fast --num_modes 1 --seed 181129): <ligand>_out.sdf
    holds the input record with new coordinates and the Uni-Dock RESULT block."""
    d, _ = inputs
    names = []
    for k, L in enumerate(synth.ligand_set(3, seed=91, heavy=(20, 30), torsions=(2, 8))):
        p = tmp_path / f"sdf{k}.sdf"
        p.write_text(L.to_sdf())
        names.append(p)
    out = tmp_path / "out"
    out.mkdir()
    r = run("--receptor", d / "rec.pdbqt", "--gpu_batch", *names, "--dir", out, "--scoring", scoring,
            "--search_mode", "fast", "--num_modes", 1, "--seed", 181129, *box_args())
    assert r.returncode == 0, r.stderr
    for p in names:
        text = (out / (p.stem + "_out.sdf")).read_text()
        assert text.count("$$$$") == 1 and text.endswith("$$$$\n")
        lines = text.split("\n")
        k = lines.index("> <Uni-Dock RESULT> ")
        score = float(lines[k + 1][len("ENERGY="):].split()[0])
        assert -20 <= score <= -1
    # --local_only on an SDF ligand writes an SDF structure (coordinates in SDF columns)
    lo = tmp_path / "local.sdf"
    r = run("--receptor", d / "rec.pdbqt", "--ligand", names[0], "--local_only", "--out", lo, *box_args())
    assert r.returncode == 0, r.stderr
    src = [l for l in names[0].read_text().splitlines() if "$$$$" not in l]
    dst = lo.read_text().splitlines()
    assert len(src) == len(dst) and all(a[30:] == b[30:] for a, b in zip(src, dst))
    assert sum(a[:30] != b[:30] for a, b in zip(src, dst)) > 0


@pytest.mark.gpu
def test_ad4_maps_written_then_read_back(inputs, tmp_path, receptor):
    """--scoring ad4 builds AutoDock maps from the receptor (charges from its
    PDBQT), --write_maps writes AutoGrid files, and --maps reads them back:
    the docking from the files equals the docking from the receptor (the maps
    are equal on the same grid, so the seeded search is too)."""
    d, names = inputs
    rec = synth.make_receptor(2000, seed=5, with_charges=True)
    (tmp_path / "recq.pdbqt").write_text(rec.to_pdbqt())
    lig = tmp_path / "lig.pdbqt"
    lig.write_text(synth.make_ligand(18, 3, seed=808, with_charges=True).to_pdbqt())
    common = ["--ligand", lig, "--scoring", "ad4", "--exhaustiveness", 8, "--max_step", 8, "--seed", 4]
    r = run("--receptor", tmp_path / "recq.pdbqt", *common, "--out", tmp_path / "a.pdbqt",
            "--write_maps", tmp_path / "maps", *box_args(16.0))
    assert r.returncode == 0, r.stderr
    for t in ("C", "OA", "HD", "e", "d"):
        assert (tmp_path / f"maps.{t}.map").exists()
    r = run("--maps", tmp_path / "maps", *common, "--out", tmp_path / "b.pdbqt")
    assert r.returncode == 0, r.stderr
    a, b = (tmp_path / "a.pdbqt").read_text(), (tmp_path / "b.pdbqt").read_text()
    ea = [float(l.split()[3]) for l in a.splitlines() if l.startswith("REMARK VINA RESULT:")]
    eb = [float(l.split()[3]) for l in b.splitlines() if l.startswith("REMARK VINA RESULT:")]
    assert ea and ea == eb


@pytest.mark.gpu
def test_paired_batch_mode(tmp_path):
    """--paired_batch_size with a JSON configuration (the reference's
    paired_batching.schema.json): every complex is its own receptor, box and
    ligand.  Each output equals a single-ligand run of that complex with the
    paired mode's settings (min_rmsd 0, energy range 3), and the score file
    holds its best affinity."""
    import json
    recs = [synth.make_receptor(1500, radius=28.0, seed=s) for s in (11, 12)]
    centers = [(0.0, 0.0, 0.0), (1.5, -1.0, 0.5)]
    cfg = {}
    for k in range(3):
        rec_path = tmp_path / f"rec{k % 2}.pdbqt"
        rec_path.write_text(recs[k % 2].to_pdbqt())
        lig_path = tmp_path / f"lig{k}.pdbqt"
        lig_path.write_text(synth.make_ligand(16 + 4 * k, 2 + k, seed=40 + k).to_pdbqt())
        c = centers[k % 2]
        if k < 2:  # .json ligand config with the box, and a key=value text config
            lc = tmp_path / f"lig{k}_config.json"
            lc.write_text(json.dumps({"center_x": c[0], "center_y": c[1], "center_z": c[2],
                                      "size_x": 20.0, "size_y": 20.0, "size_z": 20.0}))
        else:
            lc = tmp_path / f"lig{k}_config.txt"
            lc.write_text(f"center_x={c[0]}\ncenter_y={c[1]}\ncenter_z={c[2]}\n")
        cfg[f"complex{k}"] = {"protein": str(rec_path), "ligand": str(lig_path), "ligand_config": str(lc)}
    (tmp_path / "pairs.json").write_text(json.dumps(cfg))
    out = tmp_path / "out"
    out.mkdir()
    common = ["--exhaustiveness", 16, "--max_step", 8, "--seed", 5, "--num_modes", 4]
    r = run("--paired_batch_size", 2, "--ligand_index", tmp_path / "pairs.json", "--dir", out,
            "--size_x", 20, "--size_y", 20, "--size_z", 20, *common)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Found 3 to be primed." in r.stdout and "To do [2] batches" in r.stdout
    for k in range(3):
        text = (out / f"lig{k}_out.pdbqt").read_text()
        assert text.startswith("MODEL 1\nREMARK VINA RESULT:")
        best = float(text.split("\n")[1].split()[3])
        score = (out / f"lig{k}_score.txt").read_text()
        assert score.startswith("affinity(kcal/mol)[0]=")
        assert abs(float(score.split("=")[1]) - best) < 1e-3
        c = centers[k % 2]
        single = tmp_path / f"single{k}.pdbqt"
        r = run("--receptor", tmp_path / f"rec{k % 2}.pdbqt", "--ligand", tmp_path / f"lig{k}.pdbqt",
                "--center_x", c[0], "--center_y", c[1], "--center_z", c[2], "--size_x", 20, "--size_y", 20,
                "--size_z", 20, "--min_rmsd", 0, "--out", single, *common)
        assert r.returncode == 0, r.stderr
        assert single.read_text() == text


@pytest.mark.gpu
def test_bias_and_multi_bias(inputs, tmp_path):
    """--bias adds wells to the maps; --multi_bias reads <ligand>.bpf beside every
    batch ligand (and fails when one is missing)."""
    d, names = inputs
    bpf = "x y z Vset r type\n1.0 0.0 0.0 -3.0 1.2 acc\n-2.0 1.0 0.5 -2.0 1.5 map C\n"
    (tmp_path / "b.bpf").write_text(bpf)
    out = tmp_path / "biased"
    out.mkdir()
    search = ["--exhaustiveness", 16, "--max_step", 8, "--seed", 2, *box_args()]
    r = run("--receptor", d / "rec.pdbqt", "--gpu_batch", *names[:2], "--dir", out, *search, "--bias", tmp_path / "b.bpf")
    assert r.returncode == 0, r.stderr
    assert all((out / (p.stem + "_out.pdbqt")).exists() for p in names[:2])
    ligs = []
    for k, p in enumerate(names[:2]):  # copies with a .bpf beside each
        q = tmp_path / p.name
        q.write_text(p.read_text())
        q.with_suffix(".bpf").write_text(bpf)
        ligs.append(q)
    out2 = tmp_path / "multi"
    out2.mkdir()
    r = run("--receptor", d / "rec.pdbqt", "--gpu_batch", *ligs, "--dir", out2, *search, "--multi_bias")
    assert r.returncode == 0, r.stderr
    assert all((out2 / (p.stem + "_out.pdbqt")).exists() for p in ligs)
    ligs[1].with_suffix(".bpf").unlink()
    r = run("--receptor", d / "rec.pdbqt", "--gpu_batch", *ligs, "--dir", out2, *search, "--multi_bias")
    assert r.returncode != 0
