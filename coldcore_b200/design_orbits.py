"""Group-invariant covering designs: the quotient of C(v,k,t) by a
permutation group, searched as a weighted explicit-incidence cell.

Restates coldcore's ``src/coldcore/problems/perm_groups.py`` and
``design_orbits.py``:

* :class:`PermGroup`: a group on the points {0..v-1} by generators, its
  elements by closure, the permutation it induces on the colex ranks of
  r-subsets, and the orbits of r-subsets by label propagation
  (``perm_groups.py:41-144``); the built-in groups and the spec parser
  (``perm_groups.py:147-287``);
* :class:`DesignOrbits`: block orbits, t-subset orbits and the quotient
  weights w(O, U) = the number of blocks of O containing a fixed member of
  U (``design_orbits.py:52-135``).  In the quotient, cnt(U) equals the
  full cnt at every member of U and the deficiency weighted by |U| equals
  the full deficiency, so the weighted CSR engine
  (``GpuWeightedIncidenceBackend``) searches G-invariant designs;
* :func:`orbit_search`: greedy, peel and the notch descent over block
  orbits, returning the expanded block set (``design_orbits.py:218-268``).
"""
import re
import time
from itertools import combinations
from math import comb

import numpy as np

from .incidence import design_blocks, subset_ranks

#: the element list is a Python-level closure: capped
MAX_ELEMENTS = 200_000


class OrbitPartition:
    """Orbits of an index set in CSR form: ``labels`` (orbit of every
    index, numbered by smallest member), ``reps`` (smallest member),
    ``sizes``, ``starts`` and ``members`` (indices sorted by orbit)."""

    def __init__(self, size, labels):
        self.size = int(size)
        reps, inv = np.unique(np.asarray(labels), return_inverse=True)
        self.labels = inv.astype(np.int64).ravel()
        self.reps = reps.astype(np.int64)
        self.n_orbits = len(reps)
        self.sizes = np.bincount(self.labels,
                                 minlength=self.n_orbits).astype(np.int64)
        self.starts = np.concatenate(
            ([0], np.cumsum(self.sizes)[:-1])).astype(np.int64)
        self.members = np.argsort(self.labels, kind="stable").astype(np.int64)

    def orbit(self, o):
        s = int(self.starts[o])
        return self.members[s:s + int(self.sizes[o])]

    def __len__(self):
        return self.n_orbits


class PermGroup:
    """A permutation group on ``v`` points, given by generators (arrays p
    with p[x] the image of x; identities and repeats dropped)."""

    def __init__(self, v, gens=(), name=None):
        self.v = int(v)
        kept = {}
        for g in gens:
            g = np.asarray(g, dtype=np.int64).ravel()
            if len(g) != self.v or sorted(g.tolist()) != list(range(self.v)):
                raise ValueError("generator is not a permutation of 0..v-1")
            if not (g == np.arange(self.v)).all():
                kept.setdefault(g.tobytes(), g)
        self.gens = list(kept.values())
        self.name = name or "custom"
        self._elements = None

    @staticmethod
    def inverse(g):
        inv = np.empty_like(g)
        inv[g] = np.arange(len(g))
        return inv

    def join(self, other, name=None):
        if other.v != self.v:
            raise ValueError("groups on different point sets")
        return PermGroup(self.v, self.gens + other.gens,
                         name=name or f"{self.name}+{other.name}")

    def elements(self, cap=MAX_ELEMENTS):
        """Every element, by breadth-first closure from the identity."""
        if self._elements is None:
            ident = np.arange(self.v, dtype=np.int64)
            seen = {ident.tobytes(): ident}
            frontier = [ident]
            while frontier:
                nxt = []
                for e in frontier:
                    for g in self.gens:
                        h = g[e]
                        key = h.tobytes()
                        if key not in seen:
                            seen[key] = h
                            nxt.append(h)
                            if len(seen) > cap:
                                raise ValueError(f"group has more than {cap} "
                                                 "elements")
                frontier = nxt
            self._elements = list(seen.values())
        return self._elements

    def order(self, cap=MAX_ELEMENTS):
        return len(self.elements(cap))

    def induced(self, subsets):
        """Per generator, the permutation of the colex-ordered r-subsets
        (rows of ``subsets``) it induces: rank of the sorted image."""
        subsets = np.asarray(subsets, dtype=np.int64)
        out = []
        for g in self.gens:
            sig = np.empty(len(subsets), dtype=np.int64)
            step = 1 << 20
            for lo in range(0, len(subsets), step):
                img = np.sort(g[subsets[lo:lo + step]], axis=1)
                sig[lo:lo + step] = subset_ranks(img)
            out.append(sig)
        return out

    def subset_orbits(self, r, subsets=None):
        """Orbits of the r-subsets (colex ranks): every label drops to the
        minimum over its images under the generators and their inverses,
        with pointer jumping, until nothing changes."""
        n = comb(self.v, r)
        if subsets is None:
            subsets = design_blocks(self.v, r, np.arange(n, dtype=np.int64))
        lab = np.arange(n, dtype=np.int64)
        perms = self.induced(subsets)
        perms += [self.inverse(p) for p in perms]
        while True:
            before = lab.copy()
            for p in perms:
                np.minimum(lab, lab[p], out=lab)
            lab = lab[lab]
            if (lab == before).all():
                break
        return OrbitPartition(n, lab)

    def __len__(self):
        return self.order()

    def __repr__(self):
        return (f"PermGroup(v={self.v}, name={self.name!r}, "
                f"gens={len(self.gens)})")


# ------------------------------------------------------------- built-ins
def _shift(v, n_move):
    p = np.arange(v, dtype=np.int64)
    p[:n_move] = (np.arange(n_move) + 1) % n_move
    return p


def _is_prime(p):
    return p > 1 and all(p % d for d in range(2, int(p ** 0.5) + 1))


def _primitive_root(p):
    for g in range(2, p):
        x, seen = 1, set()
        for _ in range(p - 1):
            x = x * g % p
            seen.add(x)
        if len(seen) == p - 1:
            return g
    return 1


def trivial_group(v):
    return PermGroup(v, [], name="trivial")


def cyclic_group(v, fixed=0):
    """Z_{v-fixed} on the first v - fixed points."""
    n = int(v) - int(fixed)
    if n < 1:
        raise ValueError("no points left to move")
    return PermGroup(v, [_shift(v, n)],
                     name="cyclic" if not fixed else f"cyclic-{fixed}")


def dihedral_group(v):
    return PermGroup(v, [_shift(v, v), (-np.arange(v, dtype=np.int64)) % v],
                     name="dihedral")


def product_cyclic_group(a, b):
    """Z_a x Z_b on v = a b points, x = i b + j."""
    a, b = int(a), int(b)
    i, j = np.divmod(np.arange(a * b, dtype=np.int64), b)
    return PermGroup(a * b, [((i + 1) % a) * b + j, i * b + (j + 1) % b],
                     name=f"prod:{a}x{b}")


def affine_group(p, mult=None):
    """x -> a x + b mod a prime p: AGL(1,p), or the subgroup generated by
    x -> mult x and the translation."""
    p = int(p)
    if not _is_prime(p):
        raise ValueError(f"affine groups need a prime v, got {p}")
    a = _primitive_root(p) if mult is None else int(mult) % p
    if a == 0:
        raise ValueError("multiplier must be nonzero mod p")
    x = np.arange(p, dtype=np.int64)
    return PermGroup(p, [(x + 1) % p, (a * x) % p],
                     name="affine" if mult is None else f"affine:{a}")


def multiplier_group(p, mult):
    p = int(p)
    if not _is_prime(p):
        raise ValueError(f"multiplier groups need a prime v, got {p}")
    x = np.arange(p, dtype=np.int64)
    return PermGroup(p, [(int(mult) * x) % p], name=f"mult:{mult}")


_CYCLE = re.compile(r"\(([^()]*)\)")


def group_from_cycles(v, text, name=None):
    """Generators separated by ';', each a product of disjoint cycles in
    0-based labels: "(0 1 2)(3 4);(5 6)"."""
    gens = []
    for part in str(text).split(";"):
        part = part.strip()
        if not part:
            continue
        p = np.arange(v, dtype=np.int64)
        for cyc in _CYCLE.findall(part):
            pts = [int(x) for x in cyc.replace(",", " ").split()]
            if len(pts) != len(set(pts)) or any(not 0 <= x < v for x in pts):
                raise ValueError(f"bad cycle ({cyc})")
            for i, x in enumerate(pts):
                p[x] = pts[(i + 1) % len(pts)]
        gens.append(p)
    return PermGroup(v, gens, name=name or "gens")


def parse_design_group(v, spec):
    """A spec, terms joined by '+': trivial, cyclic, cyclic-N, dihedral,
    prod:AxB, affine, affine:A, mult:A, gens=<cycles> (perm_groups.py:
    242-276)."""
    v = int(v)
    G = None
    for term in str(spec).split("+"):
        term = term.strip()
        if not term:
            continue
        if term == "trivial":
            g = trivial_group(v)
        elif term == "cyclic":
            g = cyclic_group(v)
        elif term.startswith("cyclic-"):
            g = cyclic_group(v, fixed=int(term[7:]))
        elif term == "dihedral":
            g = dihedral_group(v)
        elif term.startswith("prod:"):
            a, b = (int(x) for x in term[5:].split("x"))
            if a * b != v:
                raise ValueError(f"prod:{a}x{b} needs v = {a * b}, got {v}")
            g = product_cyclic_group(a, b)
        elif term == "affine":
            g = affine_group(v)
        elif term.startswith("affine:"):
            g = affine_group(v, mult=int(term[7:]))
        elif term.startswith("mult:"):
            g = multiplier_group(v, int(term[5:]))
        elif term.startswith("gens="):
            g = group_from_cycles(v, term[5:])
        else:
            raise ValueError(f"unknown group term {term!r}")
        G = g if G is None else G.join(g, name=f"{G.name}+{g.name}")
    if G is None:
        raise ValueError("empty group spec")
    return G


def builtin_specs(v):
    """The built-in specs that apply to v."""
    out = ["cyclic", "cyclic-1", "cyclic-2", "dihedral"]
    out += [f"prod:{a}x{v // a}" for a in range(2, int(v ** 0.5) + 1)
            if v % a == 0]
    if _is_prime(v):
        out.append("affine")
    return out


# ------------------------------------------------------------ the quotient
def design_rows(v, k, t, blocks=None):
    """The C(v,k,t) incidence on the host, in the engine's layout: row c
    lists the colex ranks of block c's t-subsets, positions in lex order."""
    if blocks is None:
        blocks = design_blocks(v, k, np.arange(comb(v, k), dtype=np.int64))
    cols = [subset_ranks(blocks[:, list(s)])
            for s in combinations(range(k), t)]
    return np.stack(cols, axis=1).astype(np.int64)


class DesignOrbits:
    """Block orbits, t-subset orbits and the quotient weights of C(v,k,t)
    under a group (a :class:`PermGroup` or a spec)."""

    def __init__(self, v, k, t, group):
        self.v, self.k, self.t = int(v), int(k), int(t)
        if isinstance(group, str):
            group = parse_design_group(self.v, group)
        if not isinstance(group, PermGroup) or group.v != self.v:
            raise ValueError("group must be a PermGroup on v points")
        self.group = group
        self.order = group.order()
        blocks = design_blocks(self.v, self.k,
                               np.arange(comb(self.v, self.k), dtype=np.int64))
        self.block_part = group.subset_orbits(self.k, blocks)
        self.univ_part = group.subset_orbits(self.t)
        self.n_univ = comb(self.v, self.t)
        # pair counts P(O, U) = #{(B, T): B in O, T in U, T in B}; the
        # weight P / |U| is exact because G is transitive on U
        inc = design_rows(self.v, self.k, self.t, blocks)
        n_u = len(self.univ_part)
        keys = (self.block_part.labels[:, None] * n_u
                + self.univ_part.labels[inc]).ravel()
        uniq, counts = np.unique(keys, return_counts=True)
        orb, U = uniq // n_u, uniq % n_u
        w = counts // self.univ_part.sizes[U]
        if (w * self.univ_part.sizes[U] != counts).any():
            raise AssertionError("pair counts not divisible by |U|")
        self._O, self._U, self._w = orb, U, w.astype(np.int32)
        self._indptr = np.concatenate(([0], np.cumsum(np.bincount(
            orb, minlength=len(self.block_part))))).astype(np.int64)

    def candidate_orbits(self, short_orbits=False):
        """Orbit ids admitted as candidates: full-length ones (|O| = |G|)
        unless short orbits are asked for."""
        if short_orbits:
            return np.arange(len(self.block_part), dtype=np.int64)
        return np.flatnonzero(self.block_part.sizes == self.order)

    def quotient_csr(self, short_orbits=False):
        """(orbit ids, indptr, indices, w, uw) of the quotient incidence
        over the candidate orbits."""
        cand = self.candidate_orbits(short_orbits)
        lens = np.diff(self._indptr)[cand]
        starts = self._indptr[cand]
        pos = (np.repeat(starts - np.concatenate(([0], np.cumsum(lens)[:-1])),
                         lens) + np.arange(int(lens.sum())))
        indptr = np.concatenate(([0], np.cumsum(lens))).astype(np.int64)
        return (cand, indptr, self._U[pos].astype(np.int32), self._w[pos],
                self.univ_part.sizes.astype(np.int32))

    def expand(self, cand_idx, cand=None):
        """Quotient candidates -> sorted block indices."""
        cand = self.candidate_orbits() if cand is None else cand
        oid = cand[np.asarray(cand_idx, dtype=np.int64)]
        if not len(oid):
            return np.zeros(0, dtype=np.int64)
        return np.sort(np.concatenate([self.block_part.orbit(o) for o in oid]))

    def block_count(self, cand_idx, cand=None):
        cand = self.candidate_orbits() if cand is None else cand
        return int(self.block_part.sizes[
            cand[np.asarray(cand_idx, dtype=np.int64)]].sum())

    def summary(self):
        bs, us = self.block_part.sizes, self.univ_part.sizes
        return (f"{self.group.name} |G|={self.order}: {len(bs)} block orbits "
                f"({int((bs == self.order).sum())} full), {len(us)} t-orbits, "
                f"quotient nnz={len(self._w)}")


def quotient_backend(orbits, mu=1, short_orbits=False, backend=None,
                     **kw):
    """The quotient as a weighted incidence cell (the B200 engine's
    ``GpuWeightedIncidenceBackend`` unless another class with its
    constructor is given), with ``expand`` and ``block_count``."""
    if backend is None:
        from .incidence import GpuWeightedIncidenceBackend as backend
    cand, indptr, indices, w, uw = orbits.quotient_csr(short_orbits)
    q = backend(indptr, indices, w, len(orbits.univ_part), uw=uw, mu=mu,
                **kw)
    q.orbits, q.cand = orbits, cand
    q.expand = lambda idx: orbits.expand(idx, cand)
    q.block_count = lambda idx: orbits.block_count(idx, cand)
    return q


def orbit_search(v, k, t, group, budget_s=60.0, mu=1, seed=1,
                 short_orbits=False, floor=1, notch_budget_s=None,
                 orbits=None, backend=None, on_solved=None, reserve_s=30.0):
    """Greedy, peel and the notch descent over block orbits on the
    quotient cell.  Returns ``(blocks, searcher, quotient)``: the best
    verified G-invariant block set (sorted block indices; empty when no
    union of admitted orbits covers)."""
    from .search import Searcher
    orb = DesignOrbits(v, k, t, group) if orbits is None else orbits
    q = quotient_backend(orb, mu=mu, short_orbits=short_orbits,
                         backend=backend)
    best = {"blocks": np.zeros(0, dtype=np.int64), "n": None}

    def solved(M, idx):
        blocks = q.expand(idx)
        if best["n"] is None or len(blocks) < best["n"]:
            best["blocks"], best["n"] = blocks, len(blocks)
            if on_solved is not None:
                on_solved(len(blocks), blocks)

    s = Searcher(q, seed=seed, deadline=time.time() + budget_s + reserve_s,
                 on_solved=solved)
    # the reserve kept back from the deadline bounds the searcher's own
    s.build_reserve_s = min(s.build_reserve_s, reserve_s)
    s.loop_reserve_s = min(s.loop_reserve_s, reserve_s)
    try:
        s.load(np.zeros(0, dtype=np.int64))
        s.greedy_fill(10 ** 9)
        if s.uncov != 0:
            return best["blocks"], s, q
        nb = notch_budget_s or max(1.0, budget_s / 6)
        s.descend(floor=floor, notch_budget_s=nb, step0=1,
                  reserve_s=reserve_s, min_notch_s=min(20.0, nb))
    finally:
        if hasattr(q, "close"):
            q.close()
    return best["blocks"], s, q


def release(v, k, t, blocks, budget_s, mu=1, seed=1, floor=1,
            notch_budget_s=None, backend=None, reserve_s=30.0, step0=4):
    """Free polish of a structured start (design_orbits.py:270-298): a
    plain searcher on the full design (the engine's
    ``GpuCoveringDesignBackend`` unless another class with the signature
    (v, k, t, mu=...) is given) starts from the expanded blocks and runs
    the notch descent.  Returns ``(blocks, searcher)``."""
    from .search import Searcher
    if backend is None:
        from .incidence import GpuCoveringDesignBackend as backend
    b = backend(v, k, t, mu=mu)
    best = {"blocks": np.asarray(blocks, dtype=np.int64)}

    def solved(M, idx):
        best["blocks"] = np.asarray(idx, dtype=np.int64).copy()

    s = Searcher(b, seed=seed, deadline=time.time() + budget_s + reserve_s,
                 on_solved=solved)
    s.build_reserve_s = min(s.build_reserve_s, reserve_s)
    s.loop_reserve_s = min(s.loop_reserve_s, reserve_s)
    try:
        s.load(best["blocks"])
        if s.uncov != 0:
            raise ValueError("released solution is not feasible")
        nb = notch_budget_s or max(1.0, budget_s / 6)
        s.descend(floor=floor, notch_budget_s=nb, step0=step0,
                  reserve_s=reserve_s, min_notch_s=min(20.0, nb))
    finally:
        if hasattr(b, "close"):
            b.close()
    return best["blocks"], s
