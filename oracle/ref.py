"""Test-only ctypes wrapper of oracle/_ref/libudref.so: the reference's own CPU
sources (unidock/src/lib) built by oracle/Makefile.  Only tests, the bench's CPU
baseline leg and the smoke check call it."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libudref.so"
# the reference's source tree (oracle/Makefile's REF points into it); only the
# checkers read its own test inputs, and only when it is present
# (UD_REFERENCE_TREE, else a checkout beside this repository)
REFERENCE_TREE = Path(os.environ.get("UD_REFERENCE_TREE", Path(__file__).resolve().parents[2] / "reference"))
_lib = None


GPU_LIB = Path(__file__).resolve().parent / "_ref" / "libudref_gpu.so"
_gpu_lib = None


def gpu_available() -> bool:
    return LIB.exists() and GPU_LIB.exists()


def gpu_lib():
    """The reference's own GPU search (monte_carlo.cu, precalculate.cu) built for this GPU."""
    global _gpu_lib
    if _gpu_lib is None:
        lib()  # the GPU library resolves the reference's CPU code from libudref.so
        L = C.CDLL(str(GPU_LIB))
        L.udref_gpu_config.argtypes = [C.POINTER(C.c_void_p), C.c_int]
        L.udref_gpu_dock.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_ulonglong,
                                     C.POINTER(C.c_float), C.POINTER(C.c_double)]
        L.udref_gpu_last_error.restype = C.c_char_p
        L.udref_vina_dock.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float,
                                      C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_int]
        L.udref_parallel_mc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_uint, C.c_int, C.c_int,
                                        C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int]
        _gpu_lib = L
    return _gpu_lib


def vina_dock(receptor_path, ligand_path, center, size, spacing=0.375, exhaustiveness=8, n_poses=9, seed=0,
              threads=None):
    """The reference CLI's CPU docking of one ligand (Vina::set_receptor, set_ligand_from_file,
    compute_vina_maps, global_search; the reference's own code): energies of the modes."""
    c = np.ascontiguousarray(center, np.float32)
    s = np.ascontiguousarray(size, np.float32)
    e = np.zeros(n_poses, np.float64)
    n = gpu_lib().udref_vina_dock(str(receptor_path).encode(), str(ligand_path).encode(), _f(c), _f(s), spacing,
                                  exhaustiveness, n_poses, seed, threads or os.cpu_count(),
                                  e.ctypes.data_as(C.POINTER(C.c_double)), n_poses)
    if n < 0:
        raise RuntimeError("reference CPU docking failed")
    return e[:n]


def parallel_mc(ligand, maps, exhaustiveness, global_steps, seed=0, threads=None, n_saved=9, min_rmsd=1.0):
    """The reference's own parallel Monte-Carlo search (parallel_mc over monte_carlo::operator()) with the
    step count set to global_steps: (mode energies, mode poses) of the merged output container."""
    stride = 7 + ligand.n_torsions
    e = np.zeros(n_saved, np.float32)
    p = np.zeros((n_saved, stride), np.float32)
    n = gpu_lib().udref_parallel_mc(ligand.h, maps.h, exhaustiveness, global_steps, seed, threads or os.cpu_count(),
                                    n_saved, min_rmsd, _f(e), _f(p), stride)
    if n < 0:
        raise RuntimeError("reference parallel_mc failed")
    return e[:n], p[:n]


def gpu_bucket(ligand) -> int:
    """Size bucket (0 Small .. 4 Max) of the reference kernel that holds the ligand, or -1."""
    arr = (C.c_void_p * 1)(ligand.h)
    return gpu_lib().udref_gpu_config(arr, 1)


def gpu_dock(maps, ligands, exhaustiveness, max_step, seed):
    """The reference's GPU batched search of `ligands` (one size bucket):
    (best energy per ligand, seconds of the pair tables, seconds of do_docking, bucket)."""
    arr = (C.c_void_p * len(ligands))(*[l.h for l in ligands])
    best = np.zeros(len(ligands), np.float32)
    t = (C.c_double * 2)()
    cfg = gpu_lib().udref_gpu_dock(maps.h, arr, len(ligands), exhaustiveness, max_step, seed, _f(best), t)
    if cfg < 0:
        raise RuntimeError("reference GPU search: " + gpu_lib().udref_gpu_last_error().decode())
    return best, t[0], t[1], cfg


def reference_inputs(pattern: str) -> list[Path]:
    """The reference's own test input files matching a glob under its tree
    (empty when the tree is absent)."""
    if not REFERENCE_TREE.is_dir():
        return []
    return sorted(REFERENCE_TREE.glob(pattern))


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(LIB))
        vp, fp, ip = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_int)
        L.udref_maps_new.restype = vp
        L.udref_maps_new.argtypes = [C.c_int, fp, C.c_int, fp, ip, C.c_int, fp, fp, C.c_float, ip, C.c_int]
        L.udref_maps_free.argtypes = [vp]
        L.udref_maps_dims.argtypes = [vp, ip, fp, fp, fp]
        L.udref_maps_get.argtypes = [vp, C.c_int, fp]
        L.udref_table_fast.argtypes = [vp, C.c_int, C.c_int, C.c_float]
        L.udref_table_fast.restype = C.c_float
        L.udref_ligand_new.restype = vp
        L.udref_ligand_new.argtypes = [C.c_char_p, C.c_int, fp, C.c_int]
        L.udref_ligand_free.argtypes = [vp]
        L.udref_ligand_counts.argtypes = [vp, ip]
        L.udref_ligand_atoms.argtypes = [vp, fp, fp, ip, ip, ip, fp]
        L.udref_ligand_pairs.argtypes = [vp, ip, ip]
        L.udref_ligand_tree.argtypes = [vp, ip, ip, ip, fp]
        L.udref_initial_conf.argtypes = [vp, fp, fp, fp]
        L.udref_ligand_conf_indep.argtypes = [vp, fp]
        L.udref_eval_deriv.argtypes = [vp, vp, fp, fp, fp, C.c_float, C.c_float, fp, fp]
        L.udref_eval_deriv.restype = C.c_float
        L.udref_score.argtypes = [vp, vp, fp, fp, fp, C.c_float, fp]
        L.udref_bfgs.argtypes = [vp, vp, fp, fp, fp, C.c_float, C.c_int, ip]
        L.udref_bfgs.restype = C.c_float
        L.udref_mc.argtypes = [vp, vp, C.c_uint, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, fp, fp, C.c_int,
                               C.POINTER(C.c_longlong)]
        L.udref_nc_eval_deriv.argtypes = [vp, vp, fp, fp, fp, C.c_float, C.c_float, fp]
        L.udref_nc_eval_deriv.restype = C.c_float
        L.udref_refine.argtypes = [vp, vp, fp, fp, fp, C.c_int, fp]
        L.udref_nc_score.argtypes = [vp, vp, fp, fp, fp, C.c_float, fp]
        L.udref_cluster.argtypes = [vp, C.c_int, fp, C.c_int, fp, C.c_float, C.c_int, ip]
        L.udref_final_scores.argtypes = [vp, vp, C.c_int, fp, C.c_int, fp, C.c_int, fp]
        L.udref_maps_bias.argtypes = [vp, C.c_char_p]
        L.udref_ligand_bias.argtypes = [vp, C.c_char_p]
        L.udref_ad4_bias.argtypes = [vp, C.c_char_p]
        L.udref_ad4_map_get.argtypes = [vp, C.c_int, fp]
        L.udref_ad4_maps_read.restype = vp
        L.udref_ad4_maps_read.argtypes = [C.c_char_p, fp, C.c_int]
        L.udref_ad4_pair.argtypes = [C.c_int, C.c_float, C.c_int, C.c_float, C.c_float, fp, C.c_int]
        L.udref_ad4_pair.restype = C.c_float
        L.udref_ad4_probe.argtypes = [fp, ip, fp, C.c_int, fp, C.c_int, C.c_float, fp, C.c_int]
        L.udref_ad4_probe.restype = C.c_double
        _lib = L
    return _lib


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


VINA_W = np.array([-0.035579, -0.005156, 0.840245, -0.035069, -0.587439, 50, 5 * 0.05846 / 0.1 - 1], np.float32)
VINARDO_W = np.array([-0.045, 0.8, -0.035, -0.600, 50, 5 * 0.05846 / 0.1 - 1], np.float32)


AD4_W = np.array([0.1662, 0.1209, 0.1406, 0.1322, 50, 0.2983], np.float32)


def weights_for(sf):
    return {0: VINA_W, 1: AD4_W, 2: VINARDO_W}[sf]


def ad4_pair(t1, q1, t2, q2, r, weights=None):
    """ScoringFunction(SF_AD42)::eval of two AD-typed atoms (the reference's own code)."""
    w = np.ascontiguousarray(AD4_W if weights is None else weights, np.float32)
    return float(lib().udref_ad4_pair(int(t1), float(q1), int(t2), float(q2), float(r), _f(w), len(w)))


def ad4_probe(rec_xyz, rec_ad, rec_q, p, probe_ad, probe_q, weights=None):
    """Sum of the reference's AD4 pair energies of a probe atom at p (its map value)."""
    w = np.ascontiguousarray(AD4_W if weights is None else weights, np.float32)
    xyz = np.ascontiguousarray(rec_xyz, np.float32)
    ad = np.ascontiguousarray(rec_ad, np.int32)
    q = np.ascontiguousarray(rec_q, np.float32)
    pp = np.ascontiguousarray(p, np.float32)
    return float(lib().udref_ad4_probe(_f(xyz), _i(ad), _f(q), len(ad), _f(pp), int(probe_ad), float(probe_q),
                                       _f(w), len(w)))


class RefAd4Maps:
    """AD4 maps read by the reference's ad4cache from AutoGrid .map files."""

    def __init__(self, prefix, weights=None):
        w = np.ascontiguousarray(AD4_W if weights is None else weights, np.float32)
        self.h = lib().udref_ad4_maps_read(str(prefix).encode(), _f(w), len(w))
        if not self.h:
            raise RuntimeError("reference could not read AD4 maps " + str(prefix))

    def add_bias(self, bpf: str):
        """Bias wells added to the AD4 maps (ad4cache::set_bias)."""
        return lib().udref_ad4_bias(self.h, bpf.encode())

    def get(self, t, n):
        """The n values of map t (AD type; 35 / 36 for the electrostatic /
        desolvation map), x fastest, or None when the map is absent."""
        out = np.zeros(int(n), np.float32)
        return out if lib().udref_ad4_map_get(self.h, int(t), _f(out)) == n else None

    def __del__(self):
        if getattr(self, "h", None):
            lib().udref_maps_free(self.h)


class RefMaps:
    def __init__(self, rec_xyz, rec_xs, center, size, spacing=0.375, sf=0, types=None):
        w = weights_for(sf)
        xyz = np.ascontiguousarray(rec_xyz, np.float32)
        xs = np.ascontiguousarray(rec_xs, np.int32)
        c = np.ascontiguousarray(center, np.float32)
        s = np.ascontiguousarray(size, np.float32)
        t = np.ascontiguousarray(types if types is not None else np.arange(36), np.int32)
        self.h = lib().udref_maps_new(sf, _f(w), len(w), _f(xyz), _i(xs), len(xs), _f(c), _f(s), spacing, _i(t), len(t))
        if not self.h:
            raise RuntimeError("reference maps failed")
        self.dims = np.zeros(3, np.int32)
        self.init = np.zeros(3, np.float32)
        self.factor = np.zeros(3, np.float32)
        self.factor_inv = np.zeros(3, np.float32)
        lib().udref_maps_dims(self.h, _i(self.dims), _f(self.init), _f(self.factor), _f(self.factor_inv))

    def add_bias(self, bpf: str):
        """Bias wells added to the maps and to receptor-atom scoring (--bias)."""
        return lib().udref_maps_bias(self.h, bpf.encode())

    def get(self, xs):
        out = np.zeros(int(self.dims.prod()), np.float32)
        n = lib().udref_maps_get(self.h, int(xs), _f(out))
        if n < 0:
            return None
        return out.reshape(self.dims[2], self.dims[1], self.dims[0])

    def __del__(self):
        if getattr(self, "h", None):
            lib().udref_maps_free(self.h)


class RefLigand:
    def __init__(self, path, sf=0):
        w = weights_for(sf)
        self.h = lib().udref_ligand_new(str(path).encode(), sf, _f(w), len(w))
        if not self.h:
            raise RuntimeError("reference parse failed")
        c = np.zeros(5, np.int32)
        lib().udref_ligand_counts(self.h, _i(c))
        self.n_atoms, self.n_movable, self.n_torsions, self.n_pairs, self.n_nodes = [int(v) for v in c]

    def atoms(self):
        n = self.n_atoms
        lab = np.zeros((n, 3), np.float32)
        local = np.zeros((n, 3), np.float32)
        xs = np.zeros(n, np.int32)
        ad = np.zeros(n, np.int32)
        el = np.zeros(n, np.int32)
        q = np.zeros(n, np.float32)
        lib().udref_ligand_atoms(self.h, _f(lab), _f(local), _i(xs), _i(ad), _i(el), _f(q))
        return dict(lab=lab, local=local, xs=xs, ad=ad, el=el, charge=q)

    def pairs(self):
        a = np.zeros(max(self.n_pairs, 1), np.int32)
        b = np.zeros(max(self.n_pairs, 1), np.int32)
        lib().udref_ligand_pairs(self.h, _i(a), _i(b))
        return a[:self.n_pairs], b[:self.n_pairs]

    def tree(self):
        R = self.n_nodes
        par = np.zeros(R + 64, np.int32)
        beg = np.zeros(R + 64, np.int32)
        end = np.zeros(R + 64, np.int32)
        rel = np.zeros((R + 64, 6), np.float32)
        n = lib().udref_ligand_tree(self.h, _i(par), _i(beg), _i(end), _f(rel))
        return par[:n], beg[:n], end[:n], rel[:n]

    def conf_indep(self):
        o = np.zeros(7, np.float32)
        lib().udref_ligand_conf_indep(self.h, _f(o))
        return o

    def initial_pose(self):
        p = np.zeros(3, np.float32)
        q = np.zeros(4, np.float32)
        t = np.zeros(max(self.n_torsions, 1), np.float32)
        lib().udref_initial_conf(self.h, _f(p), _f(q), _f(t))
        return np.concatenate([p, q, t[:self.n_torsions]])

    def eval_deriv(self, maps, pose, v_intra=1000.0, v_inter=1000.0):
        pose = np.ascontiguousarray(pose, np.float32)
        p, q, t = pose[0:3].copy(), pose[3:7].copy(), np.ascontiguousarray(pose[7:].copy() if self.n_torsions else np.zeros(1, np.float32))
        g = np.zeros(6 + self.n_torsions, np.float32)
        xyz = np.zeros((self.n_atoms, 3), np.float32)
        e = lib().udref_eval_deriv(self.h, maps.h, _f(p), _f(q), _f(t), v_intra, v_inter, _f(g), _f(xyz))
        return float(e), g, xyz

    def score(self, maps, pose, v=1000.0):
        pose = np.ascontiguousarray(pose, np.float32)
        p, q, t = pose[0:3].copy(), pose[3:7].copy(), np.ascontiguousarray(pose[7:].copy() if self.n_torsions else np.zeros(1, np.float32))
        out = np.zeros(4, np.float32)
        lib().udref_score(self.h, maps.h, _f(p), _f(q), _f(t), v, _f(out))
        return out

    def bfgs(self, maps, pose, v=10.0, max_steps=None):
        pose = np.array(pose, np.float32)
        p, q = pose[0:3].copy(), pose[3:7].copy()
        t = pose[7:].copy() if self.n_torsions else np.zeros(1, np.float32)
        steps = (25 + self.n_atoms) // 3 if max_steps is None else max_steps
        ec = C.c_int()
        e = lib().udref_bfgs(self.h, maps.h, _f(p), _f(q), _f(t), v, steps, C.byref(ec))
        return float(e), np.concatenate([p, q, t[:self.n_torsions]]), ec.value

    def _split(self, pose):
        pose = np.array(pose, np.float32)
        t = pose[7:7 + self.n_torsions].copy() if self.n_torsions else np.zeros(1, np.float32)
        return pose[0:3].copy(), pose[3:7].copy(), np.ascontiguousarray(t)

    def set_bias(self, bpf: str):
        """The ligand's own wells (--multi_bias)."""
        return lib().udref_ligand_bias(self.h, bpf.encode())

    def nc_eval_deriv(self, maps, pose, slope=1e6, v=1000.0):
        """model::eval_deriv against the receptor atoms (non_cache)."""
        p, q, t = self._split(pose)
        g = np.zeros(6 + self.n_torsions, np.float32)
        e = lib().udref_nc_eval_deriv(self.h, maps.h, _f(p), _f(q), _f(t), slope, v, _f(g))
        return float(e), g

    def refine(self, maps, pose, refine_step=3):
        """The per-pose refinement of the reference's GPU search post-processing:
        (refined pose, last BFGS energy, inter against receptor atoms, intra, inside box)."""
        p, q, t = self._split(pose)
        out = np.zeros(3, np.float32)
        within = lib().udref_refine(self.h, maps.h, _f(p), _f(q), _f(t), refine_step, _f(out))
        return np.concatenate([p, q, t[:self.n_torsions]]), float(out[0]), float(out[1]), float(out[2]), bool(within)

    def nc_score(self, maps, pose, v=1000.0):
        """(inter against receptor atoms at slope 1e6, intra, intramolecular)."""
        p, q, t = self._split(pose)
        out = np.zeros(3, np.float32)
        lib().udref_nc_score(self.h, maps.h, _f(p), _f(q), _f(t), v, _f(out))
        return out

    def cluster(self, poses, energies, min_rmsd=1.0, max_modes=9):
        """Chain indices of the modes, in order, as the reference clusters chain results."""
        poses = np.ascontiguousarray(poses, np.float32)
        e = np.ascontiguousarray(energies, np.float32)
        out = np.zeros(max(len(e), 1), np.int32)
        n = lib().udref_cluster(self.h, len(e), _f(poses), poses.shape[1], _f(e), min_rmsd, max_modes, _i(out))
        return out[:n]

    def final_scores(self, maps, poses, order_e=None, receptor=True):
        """The reference's post-search scoring of this ligand's modes
        (Vina::global_search_gpu after its refinement, vina.h:232-343, score_gpu
        vina.cpp:1245-1322) from the given mode poses; `order_e` orders them
        for the choice of the intramolecular energy (Vina / Vinardo).  Rows in
        the reference's final order: [input index, total, rmsd lb, rmsd ub,
        inter + intra, inter, intra, conf-independent part, unbound]."""
        poses = np.ascontiguousarray(poses, np.float32)
        n = len(poses)
        oe = None if order_e is None else np.ascontiguousarray(order_e, np.float32)
        out = np.zeros((max(n, 1), 9), np.float32)
        k = lib().udref_final_scores(self.h, maps.h, n, _f(poses), poses.shape[1],
                                     _f(oe) if oe is not None else None, int(bool(receptor)), _f(out))
        return out[:k]

    def mc(self, maps, seed, n_chains, global_steps, local_steps=None, threads=1, hunt_cap=10.0):
        steps = (25 + self.n_atoms) // 3 if local_steps is None else local_steps
        stride = 7 + self.n_torsions
        be = np.zeros(n_chains, np.float32)
        bp = np.zeros((n_chains, stride), np.float32)
        ev = C.c_longlong()
        lib().udref_mc(self.h, maps.h, seed, n_chains, global_steps, steps, threads, hunt_cap, _f(be), _f(bp),
                       stride, C.byref(ev))
        return be, bp, ev.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().udref_ligand_free(self.h)
