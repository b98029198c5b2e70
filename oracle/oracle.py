"""ctypes wrapper of the C restatement (oracle.c) in FP32 and FP64.

Test infrastructure only: tests/, the smoke check and bench.py's CPU leg use it
as the checker of the CUDA engine.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_libs = {}

VINA_W = np.array([-0.035579, -0.005156, 0.840245, -0.035069, -0.587439, 50, 5 * 0.05846 / 0.1 - 1],
                  np.float32).astype(np.float64)
VINARDO_W = np.array([-0.045, 0.8, -0.035, -0.600, 50, 5 * 0.05846 / 0.1 - 1], np.float32).astype(np.float64)


AD4_W = np.array([0.1662, 0.1209, 0.1406, 0.1322, 50, 0.2983], np.float32).astype(np.float64)


def default_weights(sf):
    """Default weights of the scoring function (unidock/src/main/main.cpp:373-395)."""
    return {0: VINA_W, 1: AD4_W, 2: VINARDO_W}[sf]


class _Lig(C.Structure):
    _fields_ = [("n_atoms", C.c_int), ("n_nodes", C.c_int), ("n_pairs", C.c_int),
                ("local", C.c_void_p), ("node", C.c_void_p), ("gtype", C.c_void_p), ("heavy", C.c_void_p),
                ("parent", C.c_void_p), ("rel", C.c_void_p), ("pa", C.c_void_p), ("pb", C.c_void_p),
                ("ptp", C.c_void_p)]


def _grid_struct(real):
    rt = C.c_float if real == np.float32 else C.c_double

    class _Grid(C.Structure):
        _fields_ = [("dims", C.c_int * 3), ("init", rt * 3), ("factor", rt * 3), ("factor_inv", rt * 3),
                    ("dim_m1", rt * 3), ("slope", rt), ("maps", C.c_void_p)]
    return _Grid


class Oracle:
    """One precision of the restatement (np.float32 or np.float64)."""

    def __init__(self, real=np.float32):
        self.real = np.dtype(real).type
        name = "liboracle32.so" if self.real == np.float32 else "liboracle64.so"
        if name not in _libs:
            L = C.CDLL(str(HERE / "_ref" / name))
            rt = C.c_float if self.real == np.float32 else C.c_double
            vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
            L.orc_table_row.argtypes = [C.c_int, dp, C.c_int, C.c_int, C.c_int, vp, vp]
            L.orc_table_bins.argtypes = [C.c_int]
            L.orc_maps.argtypes = [C.c_int, dp, C.c_int, vp, ip, C.c_int, ip, vp, vp, ip, C.c_int, vp]
            L.orc_eval_deriv.argtypes = [vp, vp, vp, C.c_int, vp, rt, rt, vp, vp]
            L.orc_eval_deriv.restype = rt
            L.orc_eval_score.argtypes = [vp, vp, vp, C.c_int, vp, rt, vp]
            L.orc_bfgs.argtypes = [vp, vp, vp, C.c_int, vp, C.c_int, rt, ip]
            L.orc_bfgs.restype = rt
            L.orc_ad4_pair.argtypes = [C.c_int, rt, C.c_int, rt, rt, dp]
            L.orc_ad4_pair.restype = rt
            L.orc_ad4_probe.argtypes = [vp, vp, vp, C.c_int, vp, C.c_int, rt, dp]
            L.orc_ad4_probe.restype = rt
            _libs[name] = L
        self.L = _libs[name]
        self.Grid = _grid_struct(self.real)

    def _a(self, x):
        return np.ascontiguousarray(x, self.real)

    # ---- tables
    def tables(self, sf=0, weights=None):
        w = np.ascontiguousarray(default_weights(sf) if weights is None else weights, np.float64)
        nb = self.L.orc_table_bins(sf)
        ntp = 36 * 37 // 2
        fast = np.zeros((ntp, nb), self.real)
        smooth = np.zeros((ntp, nb, 2), self.real)
        for t1 in range(36):
            for t2 in range(t1, 36):
                tp = t1 + t2 * (t2 + 1) // 2
                self.L.orc_table_row(sf, w.ctypes.data_as(C.POINTER(C.c_double)), len(w), t1, t2,
                                     fast[tp].ctypes.data, smooth[tp].ctypes.data)
        return fast, smooth

    # ---- maps
    def maps(self, rec_xyz, rec_xs, dims, init, factor_inv, types, sf=0, weights=None):
        w = np.ascontiguousarray(default_weights(sf) if weights is None else weights, np.float64)
        xyz = self._a(rec_xyz)
        xs = np.ascontiguousarray(rec_xs, np.int32)
        d = np.ascontiguousarray(dims, np.int32)
        t = np.ascontiguousarray(types, np.int32)
        init_r = self._a(init)          # held: the C call reads these buffers
        finv_r = self._a(factor_inv)
        out = np.zeros((len(t), d[2], d[1], d[0]), self.real)
        self.L.orc_maps(sf, w.ctypes.data_as(C.POINTER(C.c_double)), len(w), xyz.ctypes.data,
                        xs.ctypes.data_as(C.POINTER(C.c_int)), len(xs), d.ctypes.data_as(C.POINTER(C.c_int)),
                        init_r.ctypes.data, finv_r.ctypes.data,
                        t.ctypes.data_as(C.POINTER(C.c_int)), len(t), out.ctypes.data)
        return out

    # ---- ligand / grid bundles
    def ligand(self, ex, slot_of_xs):
        """ex: dict from unidock_tools.engine.Ligand.export(); slot_of_xs maps a grid XS type to a map index."""
        fold = {19: 0, 22: 0, 25: 0, 28: 0, 20: 1, 23: 1, 26: 1, 29: 1}
        g = []
        for t in ex["xs"]:
            t = int(t)
            if t >= 36 or t in (21, 24, 27, 30):
                g.append(-1)
            else:
                g.append(slot_of_xs[fold.get(t, t)])
        keep = dict(local=self._a(ex["local"]), node=np.ascontiguousarray(ex["node"], np.int32),
                    gtype=np.array(g, np.int32), heavy=(np.asarray(ex["el"]) != 0).astype(np.int32),
                    parent=np.maximum(np.ascontiguousarray(ex["parent"], np.int32), 0),
                    rel=self._a(ex["rel"]), pa=np.ascontiguousarray(ex["pair_a"], np.int32),
                    pb=np.ascontiguousarray(ex["pair_b"], np.int32))
        xs = np.asarray(ex["xs"])
        a, b = keep["pa"], keep["pb"]
        t1, t2 = np.minimum(xs[a], xs[b]), np.maximum(xs[a], xs[b])
        keep["ptp"] = np.ascontiguousarray(t1 + t2 * (t2 + 1) // 2, np.int32)
        s = _Lig(len(ex["xs"]), len(ex["parent"]), len(a), *[keep[k].ctypes.data for k in
                                                              ("local", "node", "gtype", "heavy", "parent", "rel",
                                                               "pa", "pb", "ptp")])
        s._keep = keep
        s.n_torsions = len(ex["parent"]) - 1
        return s

    def grid(self, maps, dims, init, factor, factor_inv, slope=1e6):
        maps = self._a(maps)
        G = self.Grid()
        for i in range(3):
            G.dims[i] = int(dims[i])
            G.init[i] = float(self.real(init[i]))
            G.factor[i] = float(self.real(factor[i]))
            G.factor_inv[i] = float(self.real(factor_inv[i]))
            G.dim_m1[i] = float(self.real(int(dims[i]) - 1))
        G.slope = slope
        G.maps = maps.ctypes.data
        G._keep = maps
        return G

    def eval_deriv(self, lig, grid, smooth, pose, v_intra=1000.0, v_inter=1000.0):
        pose = self._a(pose)
        g = np.zeros(6 + lig.n_torsions, self.real)
        xyz = np.zeros((lig.n_atoms, 3), self.real)
        e = self.L.orc_eval_deriv(C.byref(lig), C.byref(grid), smooth.ctypes.data, smooth.shape[1], pose.ctypes.data,
                                  v_intra, v_inter, g.ctypes.data, xyz.ctypes.data)
        return float(e), g, xyz

    def eval_score(self, lig, grid, fast, pose, v=1000.0):
        pose = self._a(pose)
        out = np.zeros(2, self.real)
        self.L.orc_eval_score(C.byref(lig), C.byref(grid), fast.ctypes.data, fast.shape[1], pose.ctypes.data, v,
                              out.ctypes.data)
        return out

    def bfgs(self, lig, grid, smooth, pose, max_steps, v=10.0):
        x = np.array(pose, self.real, copy=True)
        ev = C.c_int()
        e = self.L.orc_bfgs(C.byref(lig), C.byref(grid), smooth.ctypes.data, smooth.shape[1], x.ctypes.data,
                            max_steps, v, C.byref(ev))
        return float(e), x, ev.value


def _ad4_weights(weights):
    return np.ascontiguousarray(AD4_W if weights is None else weights, np.float64)


def ad4_pair(oracle, t1, q1, t2, q2, r, weights=None):
    """AD4.2 pair energy of two AD-typed atoms (weights: vdW, H-bond, elec, desolv, glue)."""
    w = _ad4_weights(weights)
    return float(oracle.L.orc_ad4_pair(int(t1), float(q1), int(t2), float(q2), float(r),
                                       w.ctypes.data_as(C.POINTER(C.c_double))))


def ad4_probe(oracle, rec_xyz, rec_ad, rec_q, p, probe_ad, probe_q, weights=None):
    """Energy of a probe atom at p against every receptor atom within 20.48 A."""
    w = _ad4_weights(weights)
    xyz = oracle._a(rec_xyz)
    ad = np.ascontiguousarray(rec_ad, np.int32)
    q = oracle._a(rec_q)
    pp = oracle._a(p)
    return float(oracle.L.orc_ad4_probe(xyz.ctypes.data, ad.ctypes.data, q.ctypes.data, len(ad), pp.ctypes.data,
                                        int(probe_ad), float(probe_q), w.ctypes.data_as(C.POINTER(C.c_double))))
