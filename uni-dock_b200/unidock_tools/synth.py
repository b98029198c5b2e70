"""Seeded synthetic docking inputs.

The reference's published screening numbers use public benchmark sets that are
not available offline; these generators produce inputs with the shapes, sizes
and value distributions of the benchmark workloads instead:

* receptor: heavy atoms placed uniformly at random in a sphere by random
  sequential addition with a minimum spacing, a spherical pocket carved at the
  centre, X-Score (XS) types drawn from a fixed mix;
* ligands: random acyclic heavy-atom trees (bond length, bond angle and
  non-bonded clash rejection), element mix, polar hydrogens on N/O donors,
  a chosen number of rotatable non-terminal bonds, written as PDBQT with a
  ROOT/BRANCH torsion tree exactly as AutoDock Vina reads it
  (unidock/src/lib/parse_pdbqt.cpp:323-456, 924-960);
* poses: centre uniform in the box, uniform random unit quaternion, torsions
  uniform in (-pi, pi).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# XS type ids (unidock/src/lib/atom_constants.h:80-116)
XS = {
    "C_H": 0, "C_P": 1, "N_P": 2, "N_D": 3, "N_A": 4, "N_DA": 5, "O_P": 6, "O_D": 7,
    "O_A": 8, "O_DA": 9, "S_P": 10, "P_P": 11, "F_H": 12, "Cl_H": 13, "Br_H": 14,
    "I_H": 15, "Si": 16, "At": 17, "Met_D": 18, "W": 31,
}
XS_NAMES = {v: k for k, v in XS.items()}

# receptor XS mix of the benchmark workload
RECEPTOR_MIX = [("C_H", 0.40), ("C_P", 0.22), ("N_P", 0.08), ("N_D", 0.06), ("N_A", 0.02),
                ("O_A", 0.12), ("O_DA", 0.08), ("S_P", 0.02)]
# AutoDock type written for each receptor XS type
_REC_AD = {"C_H": "C", "C_P": "C", "N_P": "N", "N_D": "N", "N_A": "NA", "O_A": "OA",
           "O_DA": "OA", "S_P": "S"}


@dataclass
class Receptor:
    xyz: np.ndarray          # (n, 3) float32
    xs: np.ndarray           # (n,) int32 XS types
    ad: list                 # AutoDock type names
    charge: np.ndarray       # (n,) float32
    center: np.ndarray       # (3,) float32 pocket centre

    def to_pdbqt(self) -> str:
        lines = []
        for i, (p, t, q) in enumerate(zip(self.xyz, self.ad, self.charge)):
            lines.append(_pdbqt_atom("ATOM", i + 1, t, "REC", i // 10 + 1, p, float(q), t))
        return "\n".join(lines) + "\n"


def make_receptor(n_atoms: int = 3000, radius: float | None = None, min_dist: float = 3.0,
                  pocket_radius: float = 7.0, seed: int = 0, with_charges: bool = False
                  ) -> Receptor:
    """Random sequential addition of `n_atoms` points in a sphere.

    A 40 A sphere radius holds 3,000 atoms at 3.0 A spacing at a packing
    fraction of 0.16; larger receptors scale the radius with n^(1/3) so the
    density stays the same.
    """
    rng = np.random.default_rng(seed)
    if radius is None:
        radius = 40.0 * (n_atoms / 3000.0) ** (1.0 / 3.0)
    cell = min_dist
    ncell = int(math.ceil(2 * radius / cell)) + 2
    grid: dict = {}
    pts = np.empty((n_atoms, 3), dtype=np.float64)
    n = 0
    md2 = min_dist * min_dist
    tries = 0
    while n < n_atoms:
        tries += 1
        if tries > 200 * n_atoms:
            raise RuntimeError("receptor packing failed")
        p = rng.uniform(-radius, radius, 3)
        r2 = float(p @ p)
        if r2 > radius * radius or r2 < pocket_radius * pocket_radius:
            continue
        c = tuple(((p + radius) // cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in grid.get((c[0] + dx, c[1] + dy, c[2] + dz), ()):
                        d = pts[j] - p
                        if float(d @ d) < md2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        pts[n] = p
        grid.setdefault(c, []).append(n)
        n += 1
    names = [k for k, _ in RECEPTOR_MIX]
    probs = np.array([w for _, w in RECEPTOR_MIX])
    probs = probs / probs.sum()
    types = rng.choice(len(names), size=n_atoms, p=probs)
    xs = np.array([XS[names[t]] for t in types], dtype=np.int32)
    ad = [_REC_AD[names[t]] for t in types]
    charge = np.zeros(n_atoms, dtype=np.float32)
    if with_charges:
        charge = _integer_net_charges(rng, n_atoms)
    center = np.zeros(3, dtype=np.float32)
    return Receptor(pts.astype(np.float32), xs, ad, charge, center)


def _integer_net_charges(rng, n):
    q = rng.normal(0.0, 0.25, n)
    target = round(float(q.sum()))
    q += (target - q.sum()) / n
    return q.astype(np.float32)


# ---------------------------------------------------------------- ligands
_VALENCE = {"C": 4, "N": 3, "O": 2, "S": 2, "F": 1, "Cl": 1}
_ELEMENT_MIX = [("C", 0.70), ("N", 0.12), ("O", 0.14), ("F", 0.0133), ("Cl", 0.0133), ("S", 0.0134)]


@dataclass
class Ligand:
    heavy_xyz: np.ndarray            # (n, 3)
    element: list                    # element symbols
    bonds: list                      # (i, j) heavy-atom bonds of the tree
    rotatable: list                  # indices into bonds
    h_xyz: list = field(default_factory=list)     # polar hydrogens: (parent, xyz)
    charge: np.ndarray | None = None  # per heavy atom (AD4 workloads)
    name: str = "LIG"

    @property
    def n_heavy(self) -> int:
        return len(self.element)

    @property
    def n_torsions(self) -> int:
        return len(self.rotatable)

    def ad_type(self, i: int) -> str:
        e = self.element[i]
        nh = self.h_count(i)
        if e == "C":
            return "C"
        if e == "N":
            return "N" if nh > 0 else "NA"
        if e == "O":
            return "OA"
        if e == "S":
            return "SA"
        return e

    def h_count(self, i: int) -> int:
        return sum(1 for (p, _) in self.h_xyz if p == i)

    def to_pdbqt(self) -> str:
        """Vina-style PDBQT: ROOT block, nested BRANCH blocks, TORSDOF."""
        n = self.n_heavy
        adj = [[] for _ in range(n)]
        for bi, (a, b) in enumerate(self.bonds):
            adj[a].append((b, bi))
            adj[b].append((a, bi))
        rot = set(self.rotatable)
        # fragments: connected components after removing rotatable bonds
        frag = [-1] * n
        nf = 0
        for s in range(n):
            if frag[s] >= 0:
                continue
            stack = [s]
            frag[s] = nf
            while stack:
                u = stack.pop()
                for v, bi in adj[u]:
                    if bi not in rot and frag[v] < 0:
                        frag[v] = nf
                        stack.append(v)
            nf += 1
        # fragment tree; root = fragment minimising the maximum depth (most central)
        fadj = [[] for _ in range(nf)]
        for bi in rot:
            a, b = self.bonds[bi]
            fadj[frag[a]].append((frag[b], a, b))
            fadj[frag[b]].append((frag[a], b, a))

        def height(root):
            seen = {root}
            best = 0
            stack = [(root, 0)]
            while stack:
                u, d = stack.pop()
                best = max(best, d)
                for v, _, _ in fadj[u]:
                    if v not in seen:
                        seen.add(v)
                        stack.append((v, d + 1))
            return best

        sizes = [frag.count(f) for f in range(nf)]
        root = min(range(nf), key=lambda f: (height(f), -sizes[f], f))
        serial = {}
        lines = []
        counter = [0]
        charges = self.charge if self.charge is not None else np.zeros(n)
        h_of = {}
        for (p, xyz) in self.h_xyz:
            h_of.setdefault(p, []).append(xyz)

        def emit_atom(i):
            counter[0] += 1
            serial[i] = counter[0]
            t = self.ad_type(i)
            lines.append(_pdbqt_atom("ATOM", counter[0], self.element[i], self.name, 1,
                                     self.heavy_xyz[i], float(charges[i]), t))
            for hx in h_of.get(i, []):
                counter[0] += 1
                lines.append(_pdbqt_atom("ATOM", counter[0], "H", self.name, 1, hx, 0.0, "HD"))

        def frag_atoms(f, first=None):
            atoms = [i for i in range(n) if frag[i] == f]
            if first is not None:
                atoms.remove(first)
                atoms.insert(0, first)
            return atoms

        def emit_fragment(f, parent_f, first):
            for i in frag_atoms(f, first):
                emit_atom(i)
            for (g, a, b) in sorted(fadj[f], key=lambda x: x[1]):
                if g == parent_f:
                    continue
                lines.append("BRANCH %3d %3d" % (serial[a], counter[0] + 1))
                emit_fragment(g, f, b)
                lines.append("ENDBRANCH %3d %3d" % (serial[a], serial[b]))

        lines.append("REMARK  %d active torsions" % len(rot))
        lines.append("ROOT")
        for i in frag_atoms(root):
            emit_atom(i)
        lines.append("ENDROOT")
        for (g, a, b) in sorted(fadj[root], key=lambda x: x[1]):
            lines.append("BRANCH %3d %3d" % (serial[a], counter[0] + 1))
            emit_fragment(g, root, b)
            lines.append("ENDBRANCH %3d %3d" % (serial[a], serial[b]))
        lines.append("TORSDOF %d" % len(rot))
        return "\n".join(lines) + "\n"


    def to_sdf(self) -> str:
        """SDF (V2000) with the torsion-tree properties of the reference's ligand
        preparation (fragInfo, torsionInfo, atomInfo: unidock_tools
        torsion_tree.py get_sdf_torsion_tree_info): heavy atoms first, then the
        polar hydrogens; fragment 0 (the root) is the most central fragment."""
        n = self.n_heavy
        adj = [[] for _ in range(n)]
        for bi, (a, b) in enumerate(self.bonds):
            adj[a].append((b, bi))
            adj[b].append((a, bi))
        rot = set(self.rotatable)
        frag = [-1] * n
        nf = 0
        for s0 in range(n):
            if frag[s0] >= 0:
                continue
            stack = [s0]
            frag[s0] = nf
            while stack:
                u = stack.pop()
                for v, bi in adj[u]:
                    if bi not in rot and frag[v] < 0:
                        frag[v] = nf
                        stack.append(v)
            nf += 1
        fadj = [[] for _ in range(nf)]
        for bi in rot:
            a, b = self.bonds[bi]
            fadj[frag[a]].append(frag[b])
            fadj[frag[b]].append(frag[a])

        def height(root):
            seen, best, stack = {root}, 0, [(root, 0)]
            while stack:
                u, d = stack.pop()
                best = max(best, d)
                for v in fadj[u]:
                    if v not in seen:
                        seen.add(v)
                        stack.append((v, d + 1))
            return best

        sizes = [frag.count(f) for f in range(nf)]
        root = min(range(nf), key=lambda f: (height(f), -sizes[f], f))
        renum = {root: 0}
        for f in range(nf):
            if f != root:
                renum[f] = len(renum)
        charges = self.charge if self.charge is not None else np.zeros(n)
        xyz = [np.asarray(x, float) for x in self.heavy_xyz] + [np.asarray(h, float) for _, h in self.h_xyz]
        elem = list(self.element) + ["H"] * len(self.h_xyz)
        adt = [self.ad_type(i) for i in range(n)] + ["HD"] * len(self.h_xyz)
        q = [float(c) for c in charges] + [0.0] * len(self.h_xyz)
        atom_frag = [renum[frag[i]] for i in range(n)] + [renum[frag[p]] for p, _ in self.h_xyz]
        bonds = [(a, b) for a, b in self.bonds] + [(p, n + k) for k, (p, _) in enumerate(self.h_xyz)]
        out = [self.name, "  unidock_b200 synth", ""]
        out.append("%3d%3d  0  0  0  0  0  0  0  0999 V2000" % (len(xyz), len(bonds)))
        for i in range(len(xyz)):
            out.append("%10.4f%10.4f%10.4f %-3s 0  0  0  0  0  0  0  0  0  0  0  0"
                       % (xyz[i][0], xyz[i][1], xyz[i][2], elem[i]))
        for a, b in bonds:
            out.append("%3d%3d  1  0" % (a + 1, b + 1))
        out.append("M  END")
        out.append(">  <fragInfo>  (1) ")
        for f in range(nf):
            out.append(" ".join(str(i + 1) for i in range(len(xyz)) if atom_frag[i] == f))
        out.append("")
        out.append(">  <torsionInfo>  (1) ")
        for bi in sorted(rot):
            a, b = self.bonds[bi]
            out.append("%d %d %d %d" % (a + 1, b + 1, renum[frag[a]], renum[frag[b]]))
        out.append("")
        out.append(">  <atomInfo>  (1) ")
        for i in range(len(xyz)):
            out.append(str(i + 1).ljust(3) + str(q[i])[:10].ljust(10) + adt[i].ljust(2))
        out.append("")
        out.append("$$$$")
        return "\n".join(out) + "\n"


def _pdbqt_atom(rec, serial, name, resname, resseq, xyz, charge, adtype):
    nm = name if len(name) >= 4 else " " + name.ljust(3)
    return "%-6s%5d %-4s %3s A%4d    %8.3f%8.3f%8.3f%6.2f%6.2f    %6.3f %-2s" % (
        rec, serial % 100000, nm[:4], resname[:3], resseq % 10000,
        float(xyz[0]), float(xyz[1]), float(xyz[2]), 1.0, 0.0, charge, adtype)


def _rand_unit(rng):
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def _perp(u, rng):
    w = _rand_unit(rng)
    w -= u * float(w @ u)
    return w / np.linalg.norm(w)


def make_ligand(n_heavy: int, n_torsions: int, seed: int, with_charges: bool = False,
                name: str = "LIG") -> Ligand:
    """Random tree of `n_heavy` atoms grown one bond at a time.

    Bond length U(1.40, 1.54) A, bond angle 109.5 +- 5 degrees to every
    existing neighbour, non-bonded (beyond 1-3) pairs rejected under 2.5 A.
    """
    rng = np.random.default_rng(seed)
    for _attempt in range(200):
        lig = _grow_tree(n_heavy, rng)
        if lig is not None:
            break
    else:
        raise RuntimeError("ligand growth failed")
    xyz, nbr, bonds = lig
    n = n_heavy
    deg = [len(nbr[i]) for i in range(n)]
    # elements respecting degree
    elems = []
    names = [e for e, _ in _ELEMENT_MIX]
    probs = np.array([w for _, w in _ELEMENT_MIX])
    for i in range(n):
        allowed = np.array([1.0 if _VALENCE[e] >= deg[i] else 0.0 for e in names])
        p = probs * allowed
        p /= p.sum()
        elems.append(names[rng.choice(len(names), p=p)])
    # polar hydrogens on N/O with free valence, pointing away from neighbours
    hs = []
    for i in range(n):
        if elems[i] in ("N", "O"):
            free = _VALENCE[elems[i]] - deg[i]
            # keep at most one H on O, up to two on N; some N/O stay acceptor-only
            nh = min(free, 1 if elems[i] == "O" else 2)
            if elems[i] == "N" and nh > 0 and rng.random() < 0.4:
                nh = 0
            for k in range(nh):
                away = np.zeros(3)
                for j in nbr[i]:
                    away += xyz[i] - xyz[j]
                for (_, hx) in [h for h in hs if h[0] == i]:
                    away += xyz[i] - hx
                if np.linalg.norm(away) < 1e-6:
                    away = _rand_unit(rng)
                away /= np.linalg.norm(away)
                d = away + 0.35 * _perp(away, rng)
                d /= np.linalg.norm(d)
                hs.append((i, xyz[i] + 1.0 * d))
    # rotatable: non-terminal single bonds (both ends with >= 2 heavy neighbours)
    cand = [bi for bi, (a, b) in enumerate(bonds) if deg[a] >= 2 and deg[b] >= 2]
    rng.shuffle(cand)
    rot = sorted(cand[:n_torsions])
    charge = _integer_net_charges(rng, n) if with_charges else None
    return Ligand(xyz.astype(np.float64), elems, bonds, rot, hs, charge, name)


def _grow_tree(n, rng):
    xyz = np.zeros((n, 3))
    nbr = [[] for _ in range(n)]
    bonds = []
    cos_lo, cos_hi = math.cos(math.radians(114.5)), math.cos(math.radians(104.5))
    for i in range(1, n):
        placed = False
        for _try in range(400):
            j = int(rng.integers(0, i))
            if len(nbr[j]) >= 4:
                continue
            length = rng.uniform(1.40, 1.54)
            if not nbr[j]:
                d = _rand_unit(rng)
            else:
                k = nbr[j][0]
                u = xyz[k] - xyz[j]
                u /= np.linalg.norm(u)
                ang = math.radians(109.5 + rng.uniform(-5.0, 5.0))
                w = _perp(u, rng)
                d = math.cos(ang) * u + math.sin(ang) * w
            if len(nbr[j]) > 1:
                v = xyz[nbr[j]] - xyz[j]
                cosang = (v @ d) / np.linalg.norm(v, axis=1)
                if np.any(cosang < cos_lo) or np.any(cosang > cos_hi):
                    continue
            p = xyz[j] + length * d
            d2 = ((xyz[:i] - p) ** 2).sum(axis=1)
            d2[j] = 1e9
            for k in nbr[j]:
                d2[k] = 1e9
            if d2.min() < 2.5 * 2.5:
                continue
            xyz[i] = p
            nbr[j].append(i)
            nbr[i].append(j)
            bonds.append((j, i))
            placed = True
            break
        if not placed:
            return None
    xyz -= xyz.mean(axis=0)
    return xyz, nbr, bonds


def ligand_set(n: int, seed: int, heavy=(12, 48), torsions=(0, 10), dist="uniform",
               with_charges=False) -> list:
    """A seeded set of ligands with per-ligand sizes drawn as the workloads describe."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        if dist == "uniform":
            nh = int(rng.integers(heavy[0], heavy[1] + 1))
            nt = int(rng.integers(torsions[0], torsions[1] + 1))
        elif dist == "lognormal":
            nh = int(np.clip(round(rng.lognormal(math.log(28.0), 0.35)), 8, 80))
            nt = int(min(nh // 4, rng.poisson(6), 20))
        else:
            raise ValueError(dist)
        out.append(make_ligand(nh, nt, seed * 1000003 + k, with_charges, name="L%03d" % (k % 1000)))
    return out


def random_poses(n: int, n_torsions: int, box_lo, box_hi, seed: int) -> np.ndarray:
    """Poses [x, y, z, qw, qx, qy, qz, t0..] with a uniform random unit quaternion."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 7 + n_torsions), dtype=np.float32)
    out[:, 0:3] = rng.uniform(box_lo, box_hi, size=(n, 3))
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    out[:, 3:7] = q
    out[:, 7:] = rng.uniform(-math.pi, math.pi, size=(n, n_torsions))
    return out
