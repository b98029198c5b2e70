"""ctypes binding of the C ABI in include/unidock_b200.h.

This module is the Python-side mirror of the reference's docking entry points
(receptor maps, ligand parsing, fixed-pose scoring, batched search).  It loads
the in-tree ``lib/libunidock_b200.so`` and raises when it is missing: there is
no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_ROOT = Path(__file__).resolve().parent.parent      # uni-dock_b200/
# UNIDOCK_B200_LIB selects another build of the same library (e.g. a tuning variant)
LIB_PATH = Path(os.environ.get("UNIDOCK_B200_LIB", PKG_ROOT / "lib" / "libunidock_b200.so"))

SF_VINA, SF_AD4, SF_VINARDO = 0, 1, 2
UD_OK = 0
UD_ADJOINT_EXACT = 1
UD_ERR_ARG, UD_ERR_PARSE, UD_ERR_CUDA, UD_ERR_CAPACITY, UD_ERR_STATE, UD_ERR_TIMEOUT = 1, 2, 3, 4, 5, 6

_lib = None


class TuneResult(C.Structure):
    _fields_ = [("chains_per_block", C.c_int), ("lanes_per_chain", C.c_int), ("bfgs_cap", C.c_int),
                ("n_sample", C.c_int), ("n_tried", C.c_int), ("ligands_per_s", C.c_float),
                ("base_ligands_per_s", C.c_float), ("energy_shift", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class StreamConfig(C.Structure):
    _fields_ = [("slot_ligands", C.c_int), ("max_slots", C.c_int), ("ring", C.c_int), ("max_atoms", C.c_int),
                ("max_torsions", C.c_int), ("timeout_ms", C.c_int)]


class UdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"unidock_b200 error {code}: {msg}")
        self.code = code


class SearchParams(C.Structure):
    _fields_ = [
        ("exhaustiveness", C.c_int),
        ("max_step", C.c_int),
        ("num_modes", C.c_int),
        ("min_rmsd", C.c_float),
        ("energy_range", C.c_float),
        ("seed", C.c_ulonglong),
        ("form", C.c_int),
        ("chains_per_block", C.c_int),
        ("bfgs_cap", C.c_int),
        ("use_graph", C.c_int),
        ("refine_step", C.c_int),
        ("lanes_per_chain", C.c_int),
    ]


def lib():
    """Load the engine library (once)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FileNotFoundError(
            f"{LIB_PATH} is missing: build it with `make -C {PKG_ROOT}` (or __graft_entry__.build())")
    L = C.CDLL(str(LIB_PATH))
    vp, ip, fp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_float)
    sig = {
        "ud_version": ([], C.c_int),
        "ud_last_error": ([], C.c_char_p),
        "ud_receptor_parse": ([C.c_char_p, C.c_size_t, fp, ip, C.c_int, ip], C.c_int),
        "ud_maps_create": ([C.c_int, fp, C.c_int, fp, ip, C.c_int, fp, fp, C.c_float, ip, C.c_int, vp,
                            C.POINTER(vp)], C.c_int),
        "ud_maps_info": ([vp, ip, fp, fp, ip], C.c_int),
        "ud_maps_read": ([vp, C.c_int, fp, C.c_size_t], C.c_int),
        "ud_maps_destroy": ([vp], C.c_int),
        "ud_ligand_parse": ([C.c_char_p, C.c_size_t, C.POINTER(vp)], C.c_int),
        "ud_ligand_parse_sdf": ([C.c_char_p, C.c_size_t, C.c_int, C.POINTER(vp)], C.c_int),
        "ud_score_grad_receptor": ([vp, ip, fp, C.c_int, C.c_int, C.c_float, C.c_float, fp, fp, C.c_int, vp],
                                   C.c_int),
        "ud_refine": ([vp, ip, fp, C.c_int, C.c_int, C.c_int, fp, vp], C.c_int),
        "ud_batch_reset": ([vp, C.POINTER(vp), C.c_int, vp], C.c_int),
        "ud_maps_add_bias": ([vp, C.c_char_p, C.c_size_t, vp], C.c_int),
        "ud_batch_set_bias": ([vp, C.c_int, C.c_char_p, C.c_size_t], C.c_int),
        "ud_score_terms_receptor": ([vp, ip, fp, C.c_int, C.c_int, fp, vp], C.c_int),
        "ud_ligand_write": ([vp, fp, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
        "ud_ligand_counts": ([vp, ip], C.c_int),
        "ud_ligand_export": ([vp, fp, fp, ip, ip, ip, fp, ip, ip, ip, ip, fp, ip, ip], C.c_int),
        "ud_ligand_initial_pose": ([vp, fp], C.c_int),
        "ud_ligand_coords": ([vp, fp, fp], C.c_int),
        "ud_ligand_conf_indep": ([vp, fp], C.c_int),
        "ud_ligand_destroy": ([vp], C.c_int),
        "ud_batch_create": ([vp, C.POINTER(vp), C.c_int, vp, C.POINTER(vp)], C.c_int),
        "ud_batch_destroy": ([vp], C.c_int),
        "ud_score_grad": ([vp, ip, fp, C.c_int, C.c_int, C.c_float, C.c_float, fp, fp, C.c_int, vp], C.c_int),
        "ud_score_grad_device": ([vp, vp, vp, C.c_int, C.c_int, C.c_float, C.c_float, vp, vp, C.c_int, vp],
                                 C.c_int),
        "ud_score": ([vp, ip, fp, C.c_int, C.c_int, C.c_float, fp, vp], C.c_int),
        "ud_search": ([vp, C.POINTER(SearchParams), vp], C.c_int),
        "ud_search_launch": ([vp, C.POINTER(SearchParams), vp], C.c_int),
        "ud_search_prepare": ([vp, C.POINTER(SearchParams), vp], C.c_int),
        "ud_search_collect": ([vp, vp], C.c_int),
        "ud_search_chains": ([vp, fp, C.c_int, fp, ip], C.c_int),
        "ud_search_device_noalloc": ([vp, C.POINTER(SearchParams), vp, C.c_int, vp, vp, vp], C.c_int),
        "ud_stream_create": ([vp, C.POINTER(SearchParams), C.POINTER(StreamConfig), C.POINTER(vp)], C.c_int),
        "ud_stream_push": ([vp, C.POINTER(vp), C.c_int, C.POINTER(C.c_int)], C.c_int),
        "ud_stream_close": ([vp], C.c_int),
        "ud_stream_collect": ([vp, C.c_int], C.c_int),
        "ud_stream_result_count": ([vp, C.c_int, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "ud_stream_result_mode": ([vp, C.c_int, C.c_int, C.c_int, fp, fp], C.c_int),
        "ud_stream_result_write": ([vp, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_size_t,
                                    C.POINTER(C.c_size_t)], C.c_int),
        "ud_stream_chains": ([vp, C.c_int, fp, C.c_int, fp, ip], C.c_int),
        "ud_stream_finish": ([vp, C.POINTER(C.c_longlong)], C.c_int),
        "ud_stream_destroy": ([vp], C.c_int),
        "ud_result_count": ([vp, C.c_int, ip], C.c_int),
        "ud_result_mode": ([vp, C.c_int, C.c_int, fp, fp], C.c_int),
        "ud_result_write": ([vp, C.c_int, C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
        "ud_search_stats": ([vp, C.POINTER(C.c_longlong), fp], C.c_int),
        "ud_batch_upload_bytes": ([vp, C.POINTER(C.c_size_t)], C.c_int),
        "ud_optimize": ([vp, ip, fp, C.c_int, C.c_int, C.c_int, C.c_float, fp, ip, vp], C.c_int),
        "ud_device_fp32_peak": ([fp], C.c_int),
        "ud_device_l2_peak": ([fp], C.c_int),
        "ud_maps_term_count": ([vp, ip], C.c_int),
        "ud_batch_device_bytes": ([C.POINTER(vp), C.c_int, C.c_int, C.POINTER(SearchParams),
                                   C.POINTER(C.c_size_t)], C.c_int),
        "ud_ligand_parse_many": ([C.POINTER(C.c_char_p), C.POINTER(C.c_size_t), C.c_int, C.c_int, C.POINTER(vp),
                                  ip], C.c_int),
        "ud_receptor_parse_ex": ([C.c_char_p, C.c_size_t, fp, ip, ip, fp, C.c_int, ip], C.c_int),
        "ud_maps_create_ad4": ([fp, C.c_int, fp, ip, fp, C.c_int, fp, fp, C.c_float, ip, C.c_int, vp,
                                C.POINTER(vp)], C.c_int),
        "ud_maps_write": ([vp, C.c_char_p], C.c_int),
        "ud_maps_load": ([C.c_int, fp, C.c_int, C.c_char_p, vp, C.POINTER(vp)], C.c_int),
        "ud_autotune": ([vp, C.POINTER(SearchParams), C.POINTER(TuneResult), vp], C.c_int),
        "ud_maps_get_weights": ([vp, fp, C.c_int], C.c_int),
        "ud_maps_set_weights": ([vp, fp, C.c_int, vp], C.c_int),
        "ud_score_adjoint": ([vp, ip, fp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, fp, fp, C.c_int, fp,
                              C.c_int, vp], C.c_int),
        "ud_score_adjoint_device": ([vp, vp, vp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, vp, vp, C.c_int,
                                     vp, C.c_int, vp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def parse_ligands(texts, threads=0):
    """Ligands parsed on all host threads (ud_ligand_parse_many); raises on any failure."""
    bs = [t.encode() for t in texts]
    n = len(bs)
    arr = (C.c_char_p * n)(*bs)
    lens = (C.c_size_t * n)(*[len(b) for b in bs])
    out = (C.c_void_p * n)()
    status = np.zeros(n, np.int32)
    _check(lib().ud_ligand_parse_many(arr, lens, n, int(threads), out, _i(status)))
    bad = np.nonzero(status)[0]
    if len(bad):
        for h in out:
            if h:
                lib().ud_ligand_destroy(C.c_void_p(h))
        raise UdError(int(status[bad[0]]), f"{len(bad)} of {n} ligands failed to parse (first: {int(bad[0])})")
    return [Ligand("", _handle=h) for h in out]


def batch_device_bytes(ligands, sf=SF_VINA, exhaustiveness=8, num_modes=9):
    """Device bytes a batch of these ligands holds through a search
    (ud_batch_device_bytes; host-only, no GPU needed)."""
    arr = (C.c_void_p * len(ligands))(*[l.h.value for l in ligands])
    p = SearchParams(exhaustiveness, 0, num_modes, 1.0, 3.0, 0, 1, 0, 0, 0)
    out = C.c_size_t()
    _check(lib().ud_batch_device_bytes(arr, len(ligands), int(sf), C.byref(p), C.byref(out)))
    return int(out.value)


def parse_receptor_ex(text: str):
    """(xyz, xs, ad, charge) of a receptor PDBQT (ud_receptor_parse_ex)."""
    b = text.encode()
    n = C.c_int()
    _check(lib().ud_receptor_parse_ex(b, len(b), None, None, None, None, 0, C.byref(n)))
    xyz = np.zeros((n.value, 3), np.float32)
    xs = np.zeros(n.value, np.int32)
    ad = np.zeros(n.value, np.int32)
    q = np.zeros(n.value, np.float32)
    _check(lib().ud_receptor_parse_ex(b, len(b), _f(xyz), _i(xs), _i(ad), _f(q), n.value, C.byref(n)))
    return xyz, xs, ad, q


def exported_symbols():
    """Names declared in include/unidock_b200.h."""
    hdr = PKG_ROOT.parent / "include" / "unidock_b200.h"
    import re
    return sorted(set(re.findall(r"\bint\s+(ud_\w+)\s*\(", hdr.read_text())) |
                  set(re.findall(r"const char\*\s+(ud_\w+)\s*\(", hdr.read_text())))


def _check(code):
    if code != UD_OK:
        raise UdError(code, lib().ud_last_error().decode())


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def fp32_peak_tflops() -> float:
    v = C.c_float()
    _check(lib().ud_device_fp32_peak(C.byref(v)))
    return float(v.value)


def l2_peak_gbs() -> float:
    """Measured L2 read bandwidth of the current device in GB/s (ud_device_l2_peak)."""
    v = C.c_float()
    _check(lib().ud_device_l2_peak(C.byref(v)))
    return float(v.value)


def parse_receptor(pdbqt: str):
    b = pdbqt.encode()
    n = C.c_int()
    _check(lib().ud_receptor_parse(b, len(b), None, None, 0, C.byref(n)))
    xyz = np.zeros((n.value, 3), np.float32)
    xs = np.zeros(n.value, np.int32)
    _check(lib().ud_receptor_parse(b, len(b), _f(xyz), _i(xs), n.value, C.byref(n)))
    return xyz, xs


class Maps:
    """Receptor grid maps on the GPU (ud_maps_create; ud_maps_create_ad4 for
    sf=SF_AD4, where `rec_xs` holds AD types and `charges` the receptor charges)."""

    def __init__(self, rec_xyz, rec_xs, center, size, spacing=0.375, sf=SF_VINA, weights=None,
                 types=None, charges=None):
        if sf == SF_AD4:
            self._init_ad4(rec_xyz, rec_xs, charges, center, size, spacing, weights, types)
            return
        rec_xyz = np.ascontiguousarray(rec_xyz, np.float32)
        rec_xs = np.ascontiguousarray(rec_xs, np.int32)
        center = np.ascontiguousarray(center, np.float32)
        size = np.ascontiguousarray(size, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        t = None if types is None else np.ascontiguousarray(types, np.int32)
        h = C.c_void_p()
        _check(lib().ud_maps_create(sf, None if w is None else _f(w), 0 if w is None else len(w),
                                    _f(rec_xyz), _i(rec_xs), len(rec_xs), _f(center), _f(size),
                                    float(spacing), None if t is None else _i(t), 0 if t is None else len(t),
                                    None, C.byref(h)))
        self.h = h
        self.sf = sf

    def info(self):
        d = np.zeros(3, np.int32)
        init = np.zeros(3, np.float32)
        fac = np.zeros(3, np.float32)
        n = C.c_int()
        _check(lib().ud_maps_info(self.h, _i(d), _f(init), _f(fac), C.byref(n)))
        return d, init, fac, n.value

    def _init_ad4(self, rec_xyz, rec_ad, charges, center, size, spacing, weights, types):
        rec_xyz = np.ascontiguousarray(rec_xyz, np.float32)
        rec_ad = np.ascontiguousarray(rec_ad, np.int32)
        q = np.ascontiguousarray(charges, np.float32)
        center = np.ascontiguousarray(center, np.float32)
        size = np.ascontiguousarray(size, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        t = None if types is None else np.ascontiguousarray(types, np.int32)
        h = C.c_void_p()
        _check(lib().ud_maps_create_ad4(None if w is None else _f(w), 0 if w is None else len(w), _f(rec_xyz),
                                        _i(rec_ad), _f(q), len(rec_ad), _f(center), _f(size), float(spacing),
                                        None if t is None else _i(t), 0 if t is None else len(t), None,
                                        C.byref(h)))
        self.h = h
        self.sf = SF_AD4

    @classmethod
    def load(cls, prefix, sf=SF_VINA, weights=None):
        """Maps read from AutoGrid .map files (ud_maps_load, the reference's --maps)."""
        self = cls.__new__(cls)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        h = C.c_void_p()
        _check(lib().ud_maps_load(sf, None if w is None else _f(w), 0 if w is None else len(w),
                                  str(prefix).encode(), None, C.byref(h)))
        self.h = h
        self.sf = sf
        return self

    def add_bias(self, bpf: str):
        """Add AutoDock-bias style wells (BPF text) to the maps (ud_maps_add_bias, --bias)."""
        b = bpf.encode()
        _check(lib().ud_maps_add_bias(self.h, b, len(b), None))

    def write(self, prefix):
        """AutoGrid .map files <prefix>.<type>.map (ud_maps_write)."""
        _check(lib().ud_maps_write(self.h, str(prefix).encode()))

    @property
    def n_terms(self):
        n = C.c_int()
        _check(lib().ud_maps_term_count(self.h, C.byref(n)))
        return n.value

    def weights(self):
        """Current term weights (reference order; no rotatable weight)."""
        w = np.zeros(self.n_terms, np.float32)
        _check(lib().ud_maps_get_weights(self.h, _f(w), len(w)))
        return w

    def set_weights(self, w, stream=None):
        """Recombine maps and tables for new term weights on the GPU (ud_maps_set_weights)."""
        w = np.ascontiguousarray(w, np.float32)
        _check(lib().ud_maps_set_weights(self.h, _f(w), len(w), C.c_void_p(stream) if stream else None))

    def read(self, xs):
        d, _, _, _ = self.info()
        out = np.zeros(int(d.prod()), np.float32)
        _check(lib().ud_maps_read(self.h, int(xs), _f(out), out.size))
        return out.reshape(d[2], d[1], d[0])  # [z][y][x]

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ud_maps_destroy(self.h)
            self.h = None


class Ligand:
    """Host-side torsion-tree model parsed from PDBQT or SDF text
    (ud_ligand_parse; ud_ligand_parse_sdf when keep_h is given)."""

    def __init__(self, text: str, _handle=None, keep_h=None):
        if _handle is None:
            b = text.encode()
            h = C.c_void_p()
            if keep_h is None:
                _check(lib().ud_ligand_parse(b, len(b), C.byref(h)))
            else:
                _check(lib().ud_ligand_parse_sdf(b, len(b), int(bool(keep_h)), C.byref(h)))
        else:
            h = C.c_void_p(_handle)
        self.h = h
        c = np.zeros(8, np.int32)
        _check(lib().ud_ligand_counts(h, _i(c)))
        (self.n_atoms, self.n_heavy, self.n_torsions, self.n_nodes, self.n_pairs, self.torsdof,
         self.n_glue, self.local_steps) = [int(v) for v in c]

    def export(self):
        n, R, P = self.n_atoms, self.n_nodes, self.n_pairs
        out = dict(lab=np.zeros((n, 3), np.float32), local=np.zeros((n, 3), np.float32),
                   xs=np.zeros(n, np.int32), ad=np.zeros(n, np.int32), el=np.zeros(n, np.int32),
                   charge=np.zeros(n, np.float32), node=np.zeros(n, np.int32),
                   parent=np.zeros(R, np.int32), begin=np.zeros(R, np.int32), end=np.zeros(R, np.int32),
                   rel=np.zeros((R, 6), np.float32), pair_a=np.zeros(max(P, 1), np.int32),
                   pair_b=np.zeros(max(P, 1), np.int32))
        _check(lib().ud_ligand_export(self.h, _f(out["lab"]), _f(out["local"]), _i(out["xs"]), _i(out["ad"]),
                                      _i(out["el"]), _f(out["charge"]), _i(out["node"]), _i(out["parent"]),
                                      _i(out["begin"]), _i(out["end"]), _f(out["rel"]), _i(out["pair_a"]),
                                      _i(out["pair_b"])))
        out["pair_a"] = out["pair_a"][:P]
        out["pair_b"] = out["pair_b"][:P]
        return out

    def initial_pose(self):
        p = np.zeros(7 + self.n_torsions, np.float32)
        _check(lib().ud_ligand_initial_pose(self.h, _f(p)))
        return p

    def coords(self, pose):
        pose = np.ascontiguousarray(pose, np.float32)
        xyz = np.zeros((self.n_atoms, 3), np.float32)
        _check(lib().ud_ligand_coords(self.h, _f(pose), _f(xyz)))
        return xyz

    def conf_indep(self):
        o = np.zeros(7, np.float32)
        _check(lib().ud_ligand_conf_indep(self.h, _f(o)))
        return o

    def write_structure(self, pose) -> str:
        """The input record (SDF or PDBQT) with the coordinates of `pose` (ud_ligand_write)."""
        pose = np.ascontiguousarray(pose, np.float32)
        n = C.c_size_t()
        _check(lib().ud_ligand_write(self.h, _f(pose), None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value + 1)
        _check(lib().ud_ligand_write(self.h, _f(pose), buf, n.value + 1, C.byref(n)))
        return buf.value.decode()

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ud_ligand_destroy(self.h)
            self.h = None


class Batch:
    """Ligand topologies resident on the GPU (ud_batch_create)."""

    def __init__(self, maps: Maps, ligands):
        self.maps = maps
        self.ligands = list(ligands)
        arr = (C.c_void_p * len(self.ligands))(*[l.h.value for l in self.ligands])
        h = C.c_void_p()
        _check(lib().ud_batch_create(maps.h, arr, len(self.ligands), None, C.byref(h)))
        self.h = h
        self.max_torsions = max([l.n_torsions for l in self.ligands] + [0])

    def set_bias(self, lig, bpf: str):
        """Ligand `lig`'s own bias wells for receptor-atom scoring (ud_batch_set_bias, --multi_bias)."""
        b = bpf.encode()
        _check(lib().ud_batch_set_bias(self.h, int(lig), b, len(b)))

    def reset(self, ligands, stream=None):
        """Reuse this batch's handle and device buffers for other ligands
        (ud_batch_reset; the previous search must have been collected)."""
        ligands = list(ligands)
        arr = (C.c_void_p * len(ligands))(*[l.h.value for l in ligands])
        _check(lib().ud_batch_reset(self.h, arr, len(ligands), C.c_void_p(stream) if stream else None))
        self.ligands = ligands
        self.max_torsions = max([l.n_torsions for l in self.ligands] + [0])

    # ---- fixed poses
    def score_grad(self, pose_ligand, poses, v_intra=1000.0, v_inter=1000.0):
        pose_ligand = np.ascontiguousarray(pose_ligand, np.int32)
        poses = np.ascontiguousarray(poses, np.float32)
        n, stride = poses.shape
        gs = 6 + self.max_torsions
        e = np.zeros(n, np.float32)
        g = np.zeros((n, gs), np.float32)
        _check(lib().ud_score_grad(self.h, _i(pose_ligand), _f(poses), n, stride, float(v_intra),
                                   float(v_inter), _f(e), _f(g), gs, None))
        return e, g

    def score_grad_device(self, pose_ligand_ptr, poses_ptr, n, stride, e_ptr, g_ptr, g_stride,
                          v_intra=1000.0, v_inter=1000.0, stream=0):
        _check(lib().ud_score_grad_device(self.h, C.c_void_p(pose_ligand_ptr), C.c_void_p(poses_ptr), n, stride,
                                          float(v_intra), float(v_inter), C.c_void_p(e_ptr), C.c_void_p(g_ptr),
                                          g_stride, C.c_void_p(stream) if stream else None))

    def score_adjoint(self, pose_ligand, poses, v_intra=1000.0, v_inter=1000.0, exact=True, weights_grad=True):
        """Energy, pose-layout gradient (7 + T_max per pose) and term-weight
        gradient at fixed poses (ud_score_adjoint), host arrays."""
        pose_ligand = np.ascontiguousarray(pose_ligand, np.int32)
        poses = np.ascontiguousarray(poses, np.float32)
        n, stride = poses.shape
        gs = 7 + self.max_torsions
        nt = self.maps.n_terms
        e = np.zeros(n, np.float32)
        g = np.zeros((n, gs), np.float32)
        dw = np.zeros((n, nt), np.float32) if weights_grad else None
        _check(lib().ud_score_adjoint(self.h, _i(pose_ligand), _f(poses), n, stride, float(v_intra), float(v_inter),
                                      UD_ADJOINT_EXACT if exact else 0, _f(e), _f(g), gs,
                                      _f(dw) if weights_grad else None, nt, None))
        return e, g, dw

    def score_adjoint_device(self, pose_ligand_ptr, poses_ptr, n, stride, e_ptr, g_ptr=0, g_stride=0, dw_ptr=0,
                             dw_stride=0, v_intra=1000.0, v_inter=1000.0, exact=True, stream=0):
        """Device-pointer form of score_adjoint (raw addresses as ints; 0 = not wanted)."""
        _check(lib().ud_score_adjoint_device(self.h, C.c_void_p(pose_ligand_ptr), C.c_void_p(poses_ptr), n, stride,
                                             float(v_intra), float(v_inter), UD_ADJOINT_EXACT if exact else 0,
                                             C.c_void_p(e_ptr), C.c_void_p(g_ptr) if g_ptr else None, g_stride,
                                             C.c_void_p(dw_ptr) if dw_ptr else None, dw_stride,
                                             C.c_void_p(stream) if stream else None))

    # ---- receptor atoms (the reference's non_cache)
    def score_grad_receptor(self, pose_ligand, poses, slope=1e6, v=1000.0):
        """Energy and gradient against the receptor atoms (ud_score_grad_receptor)."""
        pose_ligand = np.ascontiguousarray(pose_ligand, np.int32)
        poses = np.ascontiguousarray(poses, np.float32)
        n, stride = poses.shape
        gs = 6 + self.max_torsions
        e = np.zeros(n, np.float32)
        g = np.zeros((n, gs), np.float32)
        _check(lib().ud_score_grad_receptor(self.h, _i(pose_ligand), _f(poses), n, stride, float(slope), float(v),
                                            _f(e), _f(g), gs, None))
        return e, g

    def refine(self, pose_ligand, poses, refine_step=3):
        """Refined poses and (last BFGS energy, inter, intra, inside box) per pose (ud_refine)."""
        pose_ligand = np.ascontiguousarray(pose_ligand, np.int32)
        poses = np.array(poses, np.float32, copy=True, order="C")
        n, stride = poses.shape
        out = np.zeros((n, 4), np.float32)
        _check(lib().ud_refine(self.h, _i(pose_ligand), _f(poses), n, stride, int(refine_step), _f(out), None))
        return poses, out

    def score_terms_receptor(self, pose_ligand, poses):
        """--score_only energy vector with receptor atoms (ud_score_terms_receptor)."""
        pose_ligand = np.ascontiguousarray(pose_ligand, np.int32)
        poses = np.ascontiguousarray(poses, np.float32)
        n, stride = poses.shape
        out = np.zeros((n, 8), np.float32)
        _check(lib().ud_score_terms_receptor(self.h, _i(pose_ligand), _f(poses), n, stride, _f(out), None))
        return out

    def score(self, pose_ligand, poses, v=1000.0):
        pose_ligand = np.ascontiguousarray(pose_ligand, np.int32)
        poses = np.ascontiguousarray(poses, np.float32)
        n, stride = poses.shape
        out = np.zeros((n, 2), np.float32)
        _check(lib().ud_score(self.h, _i(pose_ligand), _f(poses), n, stride, float(v), _f(out), None))
        return out

    # ---- search
    def search(self, exhaustiveness=8, max_step=0, num_modes=9, min_rmsd=1.0, energy_range=3.0, seed=0,
               form=1, chains_per_block=0, bfgs_cap=0, use_graph=0, refine_step=0, lanes_per_chain=0):
        """Search, cluster and score (ud_search).  refine_step > 0 refines the
        modes against the receptor atoms, as the reference CLI does by default
        (refine_step 3); 0 keeps the grid energies (--no_refine)."""
        p = SearchParams(exhaustiveness, max_step, num_modes, min_rmsd, energy_range, seed, form,
                         chains_per_block, bfgs_cap, use_graph, refine_step, lanes_per_chain)
        _check(lib().ud_search(self.h, C.byref(p), None))
        self.exhaustiveness = exhaustiveness

    def search_launch(self, exhaustiveness=8, max_step=0, num_modes=9, min_rmsd=1.0, energy_range=3.0, seed=0,
                      form=1, chains_per_block=0, bfgs_cap=0, use_graph=0, stream=None, refine_step=0,
                      lanes_per_chain=0):
        """Enqueue the device part only (search, clustering, refinement;
        device-resident inputs, asynchronous on `stream`, a raw cudaStream_t or
        None for the default stream)."""
        self._p = SearchParams(exhaustiveness, max_step, num_modes, min_rmsd, energy_range, seed, form,
                               chains_per_block, bfgs_cap, use_graph, refine_step, lanes_per_chain)
        _check(lib().ud_search_launch(self.h, C.byref(self._p), C.c_void_p(stream) if stream else None))
        self.exhaustiveness = exhaustiveness

    def search_device_noalloc(self, d_poses, pose_stride, d_energies, d_evals=None, stream=None, exhaustiveness=8,
                              max_step=0, seed=0, bfgs_cap=0, chains_per_block=0, lanes_per_chain=0):
        """Batched search into caller-owned device buffers (raw device
        addresses as ints), using the library's static scratch instead of
        device allocations; asynchronous on `stream` (a raw cudaStream_t or
        None for the legacy default stream).  Launch shape and BFGS cap as in
        search().  Returns per-chain results only: no clustering, and the
        batch's own result state is left untouched."""
        p = SearchParams(exhaustiveness, max_step, 9, 1.0, 3.0, seed, 1, chains_per_block, bfgs_cap, 0, 0,
                         lanes_per_chain)
        _check(lib().ud_search_device_noalloc(self.h, C.byref(p), C.c_void_p(d_poses), int(pose_stride),
                                              C.c_void_p(d_energies), C.c_void_p(d_evals) if d_evals else None,
                                              C.c_void_p(stream) if stream else None))

    def autotune(self, exhaustiveness=8, max_step=0, seed=0):
        """Pick warps per CTA, lanes per chain and the BFGS cap for this batch
        (ud_autotune); searches with chains_per_block=0, lanes_per_chain=0 and
        bfgs_cap=-1 then use them."""
        p = SearchParams(exhaustiveness, max_step, 9, 1.0, 3.0, seed, 1, 0, 0, 0)
        r = TuneResult()
        _check(lib().ud_autotune(self.h, C.byref(p), C.byref(r), None))
        return r.as_dict()

    def search_prepare(self, exhaustiveness=8, max_step=0, num_modes=9, min_rmsd=1.0, energy_range=3.0, seed=0,
                       form=1, chains_per_block=0, bfgs_cap=0, use_graph=0, stream=None, refine_step=0,
                       lanes_per_chain=0):
        """Set up a search (buffers, order, graph) without launching it (ud_search_prepare)."""
        p = SearchParams(exhaustiveness, max_step, num_modes, min_rmsd, energy_range, seed, form,
                         chains_per_block, bfgs_cap, use_graph, refine_step, lanes_per_chain)
        _check(lib().ud_search_prepare(self.h, C.byref(p), C.c_void_p(stream) if stream else None))

    def search_collect(self, stream=None):
        """Wait for the launched search, then finish and keep the modes."""
        _check(lib().ud_search_collect(self.h, C.c_void_p(stream) if stream else None))

    def optimize(self, pose_ligand, poses, v=1000.0, max_steps=0):
        pose_ligand = np.ascontiguousarray(pose_ligand, np.int32)
        poses = np.array(poses, np.float32, copy=True, order="C")
        n, stride = poses.shape
        e = np.zeros(n, np.float32)
        ev = np.zeros(n, np.int32)
        _check(lib().ud_optimize(self.h, _i(pose_ligand), _f(poses), n, stride, int(max_steps), float(v), _f(e),
                                 _i(ev), None))
        return poses, e, ev

    def chains(self):
        n = len(self.ligands) * self.exhaustiveness
        stride = 7 + self.max_torsions
        poses = np.zeros((n, stride), np.float32)
        e = np.zeros(n, np.float32)
        ev = np.zeros(n, np.int32)
        _check(lib().ud_search_chains(self.h, _f(poses), stride, _f(e), _i(ev)))
        return poses, e, ev

    def modes(self, lig):
        n = C.c_int()
        _check(lib().ud_result_count(self.h, lig, C.byref(n)))
        out = []
        for k in range(n.value):
            pose = np.zeros(7 + self.ligands[lig].n_torsions, np.float32)
            en = np.zeros(8, np.float32)
            _check(lib().ud_result_mode(self.h, lig, k, _f(pose), _f(en)))
            out.append((pose, en))
        return out

    def write(self, lig, fmt=0):
        ln = C.c_size_t()
        _check(lib().ud_result_write(self.h, lig, fmt, None, 0, C.byref(ln)))
        buf = C.create_string_buffer(ln.value + 1)
        _check(lib().ud_result_write(self.h, lig, fmt, buf, ln.value + 1, C.byref(ln)))
        return buf.value.decode()

    def upload_bytes(self):
        """Host-to-device bytes of the last topology upload (ud_batch_upload_bytes)."""
        n = C.c_size_t()
        _check(lib().ud_batch_upload_bytes(self.h, C.byref(n)))
        return int(n.value)

    def stats(self):
        ev = C.c_longlong()
        ms = C.c_float()
        _check(lib().ud_search_stats(self.h, C.byref(ev), C.byref(ms)))
        return ev.value, ms.value

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ud_batch_destroy(self.h)
            self.h = None


class Stream:
    """Streaming screen (ud_stream_*): one persistent search kernel, launched
    at creation, fed slot by slot with push(); collect(slot) waits for a
    slot's chains and finishes its modes.  Slot s may be pushed once slot
    s - ring was collected."""

    def __init__(self, maps: Maps, exhaustiveness=8, max_step=20, num_modes=9, min_rmsd=1.0, energy_range=3.0,
                 seed=0, refine_step=0, bfgs_cap=0, chains_per_block=0, slot_ligands=64, max_slots=64, ring=2,
                 max_atoms=64, max_torsions=16, timeout_ms=0):
        self.maps = maps
        self.exhaustiveness = exhaustiveness
        self.max_torsions = max_torsions
        self._p = SearchParams(exhaustiveness, max_step, num_modes, min_rmsd, energy_range, seed, 1,
                               chains_per_block, bfgs_cap, 0, refine_step, 0)
        cfg = StreamConfig(slot_ligands, max_slots, ring, max_atoms, max_torsions, timeout_ms)
        h = C.c_void_p()
        _check(lib().ud_stream_create(maps.h, C.byref(self._p), C.byref(cfg), C.byref(h)))
        self.h = h
        self.slots = {}

    def push(self, ligands):
        ligands = list(ligands)
        arr = (C.c_void_p * len(ligands))(*[l.h.value for l in ligands])
        k = C.c_int()
        _check(lib().ud_stream_push(self.h, arr, len(ligands), C.byref(k)))
        self.slots[k.value] = ligands
        return k.value

    def close(self):
        _check(lib().ud_stream_close(self.h))

    def collect(self, slot):
        _check(lib().ud_stream_collect(self.h, int(slot)))

    def chains(self, slot):
        n = len(self.slots[slot]) * self.exhaustiveness
        stride = 7 + self.max_torsions
        poses = np.zeros((n, stride), np.float32)
        e = np.zeros(n, np.float32)
        ev = np.zeros(n, np.int32)
        _check(lib().ud_stream_chains(self.h, int(slot), _f(poses), stride, _f(e), _i(ev)))
        return poses, e, ev

    def modes(self, slot, lig):
        n = C.c_int()
        _check(lib().ud_stream_result_count(self.h, int(slot), int(lig), C.byref(n)))
        out = []
        for k in range(n.value):
            pose = np.zeros(7 + self.slots[slot][lig].n_torsions, np.float32)
            en = np.zeros(8, np.float32)
            _check(lib().ud_stream_result_mode(self.h, int(slot), int(lig), k, _f(pose), _f(en)))
            out.append((pose, en))
        return out

    def write(self, slot, lig, fmt=0):
        ln = C.c_size_t()
        _check(lib().ud_stream_result_write(self.h, int(slot), int(lig), fmt, None, 0, C.byref(ln)))
        buf = C.create_string_buffer(ln.value + 1)
        _check(lib().ud_stream_result_write(self.h, int(slot), int(lig), fmt, buf, ln.value + 1, C.byref(ln)))
        return buf.value.decode()

    def finish(self):
        ev = C.c_longlong()
        _check(lib().ud_stream_finish(self.h, C.byref(ev)))
        return ev.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().ud_stream_destroy(self.h)
            self.h = None
