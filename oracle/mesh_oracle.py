"""CPU restatement of the reference mesh propagation -- TEST INFRASTRUCTURE.

This file is the checker for the library's mesh driver (gpv_mesh_drive /
gpv_mesh_solve).  Only the tests, the smoke check and the benchmark's CPU
baseline leg use it; the library never does.

It restates, in plain Python, the propagation stage of the reference's
Mesh::solve_impl (src/mesh.rs:628-764) in the reference's own structure:

* connectivity (:1705-1772), Adjacency (:1838-1872)
* find_seed_node (:1682-1690)
* solve_node, two attempts (:1068-1106)
* solve_neighbours_from, the serial RG cascade (:1112-1154, :683-705)
* expand_parallel + greedy_graph_colour, layer-RG rounds (:1169-1252,
  :1884-1903, :706-764)
* precondition_warp / affine_field_fit / ols_solve / project_warp
  (:2101-2233), with the normal-equation inverse done as the reference's
  linear-algebra crate (nalgebra) does it: cofactors for a 3x3 matrix
  (exact-zero determinant = singular), LU with partial pivoting and a
  unit-lower / upper triangular solve otherwise (exact-zero pivot =
  singular).
* store_result (:2385-2402)

A colour's subsets are independent (no two share an element), so each colour
is solved as one call of the batch `solver` here too; that is exactly the
reference's rayon par_iter over the colour, folded in ascending node order.
The corrections stage (:766-790) is not part of the path and not restated.

`solver(desc, tolerance) -> results` takes a DESC_DTYPE array and returns a
RESULT_DTYPE array (oracle.solve_batch fits).
"""
from __future__ import annotations

import heapq
import struct

import numpy as np

EMPTY_MASK, FEATURELESS, SINGULAR_H, SINGULAR_WDELTA, TIMEOUT, CANCELLED, INVALID_SUBSET = 1, 2, 3, 4, 6, 7, 8
_FATAL = {EMPTY_MASK: "empty subset mask", FEATURELESS: "featureless subset", SINGULAR_H: "singular Hessian",
          SINGULAR_WDELTA: "singular warp increment", TIMEOUT: "timed out", CANCELLED: "cancelled",
          INVALID_SUBSET: "invalid subset"}
_SIDES = {0: (3, 5), 1: (3, 4), 2: (4, 5), 3: (0, 1), 4: (1, 2), 5: (0, 2)}


class Cancelled(Exception):
    """The progress observer asked to stop (src/error.rs Cancelled)."""


def connectivity(elements, mesh_order, idx, full=False):
    """src/mesh.rs:1705-1772 (brute-force scan, sorted unique)."""
    out = set()
    for row in elements:
        row = [int(v) for v in row]
        if mesh_order == 1 or full:
            if idx in row:
                out.update(v for v in row if v != idx)
        else:
            for col, v in enumerate(row):
                if v == idx:
                    out.update(row[j] for j in _SIDES[col] if row[j] != idx)
    return sorted(out)


def adjacency(elements, mesh_order, n_nodes):
    """Adjacency::build (src/mesh.rs:1847-1863): per node (full, edge)."""
    incident = [[] for _ in range(n_nodes)]
    for e, row in enumerate(elements):
        for v in row:
            incident[int(v)].append(e)
    full, edge = [], []
    for i in range(n_nodes):
        f, g = set(), set()
        for e in incident[i]:
            row = [int(v) for v in elements[e]]
            f.update(v for v in row if v != i)
            if mesh_order == 2:
                for col, v in enumerate(row):
                    if v == i:
                        g.update(row[j] for j in _SIDES[col] if row[j] != i)
        full.append(sorted(f))
        edge.append(sorted(g) if mesh_order == 2 else sorted(f))
    return full, edge


def find_seed_node(nodes, coord):
    """src/mesh.rs:1682-1690: the first node at the least squared distance."""
    best, best_d = 0, None
    for i in range(len(nodes)):
        dx = nodes[i][0] - coord[0]
        dy = nodes[i][1] - coord[1]
        d = dx * dx + dy * dy
        if best_d is None or d < best_d:
            best, best_d = i, d
    return best


def greedy_graph_colour(full, candidates):
    """src/mesh.rs:1884-1903 (candidates sorted ascending)."""
    pos = {c: k for k, c in enumerate(candidates)}
    colour = [None] * len(candidates)
    for i, c in enumerate(candidates):
        used = set()
        for nb in full[c]:
            k = pos.get(nb)
            if k is not None and colour[k] is not None:
                used.add(colour[k])
        k = 0
        while k in used:
            k += 1
        colour[i] = k
    return colour


def project_warp(p, dx, dy):
    """src/mesh.rs:2101-2122: Taylor expansion of the warp over (dx, dy)."""
    q = list(p)
    if len(p) >= 6:
        q[0] = p[0] + p[2] * dx + p[4] * dy
        q[1] = p[1] + p[3] * dx + p[5] * dy
    if len(p) >= 12:
        q[0] += 0.5 * p[6] * dx * dx + p[8] * dx * dy + 0.5 * p[10] * dy * dy
        q[1] += 0.5 * p[7] * dx * dx + p[9] * dx * dy + 0.5 * p[11] * dy * dy
        q[2] = p[2] + p[6] * dx + p[8] * dy
        q[3] = p[3] + p[7] * dx + p[9] * dy
        q[4] = p[4] + p[8] * dx + p[10] * dy
        q[5] = p[5] + p[9] * dx + p[11] * dy
    return q


def _inverse(a):
    """Matrix inverse as nalgebra's try_inverse computes it; None if singular."""
    m = len(a)
    if m == 3:
        m11, m12, m13 = a[0]
        m21, m22, m23 = a[1]
        m31, m32, m33 = a[2]
        minor_22_33 = m22 * m33 - m32 * m23
        minor_21_33 = m21 * m33 - m31 * m23
        minor_21_32 = m21 * m32 - m31 * m22
        det = m11 * minor_22_33 - m12 * minor_21_33 + m13 * minor_21_32
        if det == 0.0:
            return None
        return [[minor_22_33 / det, (m13 * m32 - m33 * m12) / det, (m12 * m23 - m22 * m13) / det],
                [-minor_21_33 / det, (m11 * m33 - m31 * m13) / det, (m13 * m21 - m23 * m11) / det],
                [minor_21_32 / det, (m12 * m31 - m32 * m11) / det, (m11 * m22 - m21 * m12) / det]]
    lu = [list(r) for r in a]
    perm = list(range(m))
    for i in range(m):
        piv = i
        for r in range(i + 1, m):
            if abs(lu[r][i]) > abs(lu[piv][i]):
                piv = r
        if lu[piv][i] == 0.0:
            return None
        if piv != i:
            lu[i], lu[piv] = lu[piv], lu[i]
            perm[i], perm[piv] = perm[piv], perm[i]
        for r in range(i + 1, m):
            lu[r][i] /= lu[i][i]
            f = lu[r][i]
            for c in range(i + 1, m):
                lu[r][c] -= f * lu[i][c]
    inv = [[0.0] * m for _ in range(m)]
    for c in range(m):
        b = [1.0 if perm[r] == c else 0.0 for r in range(m)]
        for k in range(m):  # unit lower, column oriented
            for r in range(k + 1, m):
                b[r] -= lu[r][k] * b[k]
        for k in range(m - 1, -1, -1):  # upper, column oriented
            b[k] /= lu[k][k]
            for r in range(k):
                b[r] -= lu[r][k] * b[k]
        for r in range(m):
            inv[r][c] = b[r]
    return inv


def ols_solve(rows, y):
    """src/mesh.rs:2220-2233: (A^T A)^-1 A^T y, None when A^T A is singular."""
    m = len(rows[0])
    ata = [[_dot([rows[r][i] for r in range(len(rows))], [rows[r][j] for r in range(len(rows))]) for j in range(m)]
           for i in range(m)]
    aty = [_dot([rows[r][i] for r in range(len(rows))], y) for i in range(m)]
    inv = _inverse(ata)
    if inv is None:
        return None
    return [_dot(inv[i], aty) for i in range(m)]


def _dot(a, b):
    # plain left-to-right accumulation (the built-in sum() of Python >= 3.12
    # compensates its rounding, which a matrix product does not)
    s = 0.0
    for x, y in zip(a, b):
        s += x * y
    return s


def affine_field_fit(nodes, target, trusted, p, p_len):
    """src/mesh.rs:2170-2215."""
    quad = p_len >= 12 and len(trusted) >= 6
    rows = []
    for i in trusted:
        dx = nodes[i][0] - target[0]
        dy = nodes[i][1] - target[1]
        rows.append([1.0, dx, dy, dx * dx, dx * dy, dy * dy] if quad else [1.0, dx, dy])
    cu = ols_solve(rows, [p[i][0] for i in trusted])
    if cu is None:
        return None
    cv = ols_solve(rows, [p[i][1] for i in trusted])
    if cv is None:
        return None
    w = [0.0] * p_len
    w[0], w[1], w[2], w[3], w[4], w[5] = cu[0], cv[0], cu[1], cv[1], cu[2], cv[2]
    if quad:
        w[6], w[7], w[8], w[9], w[10], w[11] = 2.0 * cu[3], 2.0 * cv[3], cu[4], cv[4], 2.0 * cu[5], 2.0 * cv[5]
    return w


def precondition_warp(nodes, target, trusted, c_zncc, p, p_len):
    """src/mesh.rs:2130-2151."""
    if len(trusted) >= 3:
        fit = affine_field_fit(nodes, target, trusted, p, p_len)
        if fit is not None:
            return fit
    if trusted:
        best = trusted[0]
        for i in trusted[1:]:  # Iterator::max_by keeps the last of equal maxima
            if c_zncc[i] >= c_zncc[best]:
                best = i
        return project_warp(list(p[best][:p_len]), target[0] - nodes[best][0], target[1] - nodes[best][1])
    return [0.0] * p_len


def _key(c):
    return struct.unpack("<Q", struct.pack("<d", c))[0]


def solve_mesh(nodes, elements, solver, *, seed_coord, radius, subset_order=1, seed_warp=None, seed_tolerance=0.9,
               tolerance=0.75, preconditioning="RG", batch_factor=4, root_rel_eps=0.02, max_workers=1,
               progress=None, desc_dtype=None):
    """Propagation stage of Mesh::solve_impl (src/mesh.rs:628-764).

    Returns dict(results, rounds, seed_node, quality_ok, c_zncc, p, stats).
    Raises ValueError for a subset the reference rejects (Err / panic) and
    Cancelled when progress(done, total) returns True.
    """
    nodes = [(float(x), float(y)) for x, y in np.asarray(nodes, dtype=np.float64)]
    elements = np.asarray(elements, dtype=np.int64)
    n = len(nodes)
    mesh_order = 2 if elements.shape[1] == 6 else 1
    p_len = 6 * subset_order
    full, edge = adjacency(elements, mesh_order, n)
    stored, propagated = [False] * n, [False] * n
    quality_ok, c_zncc = [False] * n, [0.0] * n
    p = [[0.0] * 12 for _ in range(n)]
    results = [None] * n
    rounds = [-1] * n
    heap = []
    st = dict(batches=0, solves=0, retries=0)
    state = dict(done=0, round=0)

    def call(ids, warps, tol):
        d = np.zeros(len(ids), desc_dtype)
        for k, (i, w) in enumerate(zip(ids, warps)):
            d[k]["coord"] = nodes[i]
            d[k]["p0"][:len(w)] = w
            d[k]["order"] = subset_order
            d[k]["radius"] = radius
        st["batches"] += 1
        st["solves"] += len(ids)
        r = solver(d, tol)
        for k, i in enumerate(ids):
            s = int(r[k]["status"])
            if s in _FATAL:
                raise ValueError(f"mesh node {i}: {_FATAL[s]}")
        return r

    def solve_nodes(ids, warps, tol):  # solve_node (:1068-1106) for independent nodes
        ra = call(ids, warps, tol)
        out = [ra[k].copy() for k in range(len(ids))]
        retry = [k for k in range(len(ids)) if not ra[k]["quality_ok"] and any(v != 0.0 for v in warps[k])]
        if retry:
            st["retries"] += len(retry)
            rb = call([ids[k] for k in retry], [[0.0] * p_len for _ in retry], tol)
            for t, k in enumerate(retry):
                if rb[t]["quality_ok"] or rb[t]["c_zncc"] > ra[k]["c_zncc"]:
                    out[k] = rb[t].copy()
        return out

    def store(i, r):  # store_result (:2385-2402) + node_done
        quality_ok[i] = bool(r["quality_ok"])
        c = float(r["c_zncc"])
        c_zncc[i] = 0.0 if c != c else max(c, 0.0)
        p[i] = [float(v) for v in r["p"][:p_len]] + [0.0] * (12 - p_len)
        results[i] = r
        rounds[i] = state["round"]
        stored[i] = True
        state["done"] += 1
        if progress is not None and progress(state["done"], n):
            raise Cancelled()

    def push(i):
        heapq.heappush(heap, (-_key(c_zncc[i]), -i))

    def pop():
        k, i = heapq.heappop(heap)
        return -k, -i

    def trusted_of(i):
        return [t for t in full[i] if stored[t] and quality_ok[t]]

    def neighbours_from(cur):  # :1112-1154
        for nb in edge[cur]:
            if stored[nb]:
                continue
            w = precondition_warp(nodes, nodes[nb], trusted_of(nb), c_zncc, p, p_len)
            r = solve_nodes([nb], [w], tolerance)[0]
            store(nb, r)
            push(nb)
            state["round"] += 1

    def expand(roots):  # :1169-1252
        cand = sorted({nb for r in roots for nb in edge[r] if not stored[nb]})
        if not cand:
            return
        colour = greedy_graph_colour(full, cand)
        for c in range(max(colour) + 1):
            ids = [cand[k] for k in range(len(cand)) if colour[k] == c]
            warps = [precondition_warp(nodes, nodes[i], trusted_of(i), c_zncc, p, p_len) for i in ids]
            res = solve_nodes(ids, warps, tolerance)
            for i, r in zip(ids, res):
                store(i, r)
                push(i)
            state["round"] += 1

    seed = find_seed_node(nodes, seed_coord)
    sw = list(seed_warp if seed_warp is not None else [])[:p_len]
    sw += [0.0] * (p_len - len(sw))
    store(seed, solve_nodes([seed], [sw], seed_tolerance)[0])
    state["round"] += 1
    propagated[seed] = True
    push(seed)
    if preconditioning == "RG":
        neighbours_from(seed)
        while heap:
            _, cur = pop()
            if propagated[cur]:
                continue
            propagated[cur] = True
            neighbours_from(cur)
    elif preconditioning == "layer-RG":
        root_cap = max(1, batch_factor) * max(1, max_workers)
        expand([seed])
        while heap:
            top_key, top = pop()
            if propagated[top]:
                continue
            propagated[top] = True
            roots = [top]
            threshold = struct.unpack("<d", struct.pack("<Q", top_key))[0] * (1.0 - root_rel_eps)
            while len(roots) < root_cap and heap:
                k = struct.unpack("<d", struct.pack("<Q", -heap[0][0]))[0]
                if not k >= threshold:
                    break
                _, r = pop()
                if propagated[r]:
                    continue
                propagated[r] = True
                roots.append(r)
            expand(roots)
    else:
        raise ValueError(f"preconditioning must be 'RG' or 'layer-RG', got {preconditioning!r}")
    st["rounds"] = state["round"]
    st["n_unreached"] = sum(1 for s in stored if not s)
    st["n_bad"] = sum(1 for q in quality_ok if not q)
    return dict(results=results, rounds=np.array(rounds), seed_node=seed, quality_ok=np.array(quality_ok),
                c_zncc=np.array(c_zncc), p=np.array(p), stats=st)
