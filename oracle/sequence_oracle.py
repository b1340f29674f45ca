"""CPU restatement of the reference sequence loop -- TEST INFRASTRUCTURE.

Checker for gpv.Sequence (only tests use it).  Restates, in plain Python:

* Sequence::solve's pair loop (src/sequence.rs:624-968): reference-update
  fallback for a failed non-consecutive pair (:806-818), curtailment for a
  failed consecutive pair (:819-838), the override retry (tolerance 0 and no
  quality gate, :755-766) and its log (:859-865), sequential reference
  updates (:940-952), seed guidance (:922-937);
* deformation_preconditioning (src/sequence.rs:1062-1097) through the
  particle's mesh path: element_locator (src/particle.rs:968-1018),
  local_coordinates / det3 (:135-183), shape_function (:194-236),
  warp_increment (:254-316), strain clipping (:1426-1434);
* each pair's Mesh::solve as oracle/mesh_oracle.py's propagation over the FP64
  oracle, with the quality gate (src/mesh.rs:792-799) applied to it.
"""
from __future__ import annotations

import mesh_oracle as MO


def _det3(a00, a01, a02, a10, a11, a12, a20, a21, a22):
    return a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20)


def local_coordinates(coord, nodes3):
    px, py = coord
    (n0x, n0y), (n1x, n1y), (n2x, n2y) = nodes3[0], nodes3[1], nodes3[2]
    den = _det3(1.0, 1.0, 1.0, n0x, n1x, n2x, n0y, n1y, n2y)
    z = _det3(1.0, 1.0, 1.0, px, n1x, n2x, py, n1y, n2y) / den
    e = _det3(1.0, 1.0, 1.0, px, n2x, n0x, py, n2y, n0y) / den
    return z, e, 1.0 - z - e, den


def _shape(order, z, e, t):
    if order == 1:
        return [z, e, t], [[1.0, 0.0, -1.0], [0.0, 1.0, -1.0]], None
    n = [z * (2 * z - 1), e * (2 * e - 1), t * (2 * t - 1), 4 * z * e, 4 * e * t, 4 * t * z]
    dn = [[4 * z - 1, 0.0, 1 - 4 * t, 4 * e, -4 * e, 4 * (t - z)],
          [0.0, 4 * e - 1, 1 - 4 * t, 4 * z, 4 * (t - e), -4 * z]]
    d2n = [[4.0, 0, 4, 0, 0, -8], [0, 0, 4, 4, -4, -4], [0, 4, 4, 0, -8, 0]]
    return n, dn, d2n


def _mat(a, b):
    return [[sum(a[i][k] * b[k][j] for k in range(len(b))) for j in range(len(b[0]))] for i in range(len(a))]


def warp_increment(coord, x, u, order):
    z, e, t, den = local_coordinates(coord, x)
    n, dn, d2n = _shape(order, z, e, t)
    w = [0.0] * (6 * order)
    w[0] = sum(n[k] * u[k][0] for k in range(len(n)))
    w[1] = sum(n[k] * u[k][1] for k in range(len(n)))
    jx, ju = _mat(dn, x), _mat(dn, u)
    det = jx[0][0] * jx[1][1] - jx[0][1] * jx[1][0]
    inv = [[jx[1][1] / det, -jx[0][1] / det], [-jx[1][0] / det, jx[0][0] / det]]
    g = _mat(inv, ju)
    w[2], w[3], w[4], w[5] = g[0][0], g[0][1], g[1][0], g[1][1]
    if order == 2:
        d00, d01 = (x[1][1] - x[2][1]) / den, (x[2][1] - x[0][1]) / den
        d10, d11 = (x[2][0] - x[1][0]) / den, (x[0][0] - x[2][0]) / den
        kxi = [[d00 * d00, 2 * d00 * d01, d01 * d01], [d00 * d10, d00 * d11 + d01 * d10, d01 * d11],
               [d10 * d10, 2 * d10 * d11, d11 * d11]]
        h = _mat(kxi, _mat(d2n, u))
        w[6:12] = [h[0][0], h[0][1], h[1][0], h[1][1], h[2][0], h[2][1]]
    return w


def element_locator(coord, nodes, elements):
    cents = []
    for idx, el in enumerate(elements):
        cx = (nodes[el[0]][0] + nodes[el[1]][0] + nodes[el[2]][0]) / 3.0
        cy = (nodes[el[0]][1] + nodes[el[1]][1] + nodes[el[2]][1]) / 3.0
        cents.append(((cx - coord[0]) ** 2 + (cy - coord[1]) ** 2, idx))
    cents.sort(key=lambda c: c[0])  # a stable sort, as sort_by
    for _, idx in cents:
        el = elements[idx]
        z, e, t, _ = local_coordinates(coord, [nodes[el[0]], nodes[el[1]], nodes[el[2]]])
        if z >= 0.0 and e >= 0.0 and t >= 0.0:
            return idx, False
    return cents[0][1], True


def deformation_preconditioning(nodes, elements, disps, seed_coord, mesh_order, subset_order):
    nodes = [[float(a), float(b)] for a, b in nodes]
    elements = [[int(v) for v in row] for row in elements]
    idx, _ = element_locator(seed_coord, nodes, elements)
    el = elements[idx]
    w = warp_increment(seed_coord, [nodes[k] for k in el], [[float(disps[k][0]), float(disps[k][1])] for k in el],
                       mesh_order)
    for k in range(2, len(w)):
        w[k] = min(max(w[k], -0.99), 0.99)
    out = [0.0] * (6 * subset_order)
    k = 6 * min(mesh_order, subset_order)
    out[:k] = w[:k]
    return w[:2], out


def solve_sequence(frames_c, shape, border, nodes, elements, solver_for, *, radius, seed_coord, seed_warp=None,
                   seed_tolerance=0.9, tolerance=0.75, subset_order=1, guide=True, sequential=False, override=False,
                   desc_dtype=None, **mesh_kw):
    """frames_c: per frame the oracle coefficients; solver_for(Cf, Cg) -> solver(desc, tol)."""
    n_images = len(frames_c)
    n_pairs = n_images - 1
    mesh_order = 2 if len(elements[0]) == 6 else 1
    seed_coord = [float(seed_coord[0]), float(seed_coord[1])]
    sw = [0.0] * (6 * subset_order)
    for k, v in enumerate(list(seed_warp or [])[:len(sw)]):
        sw[k] = float(v)
    f_index, g_index = 0, 1
    pairs, override_log, reference_updates = [], [], [False] * n_pairs
    mesh_override = pending = unsolvable = False
    while True:
        tol = 0.0 if mesh_override else tolerance
        sol = MO.solve_mesh(nodes, elements, solver_for(frames_c[f_index], frames_c[g_index]), radius=radius,
                            seed_coord=tuple(seed_coord), seed_warp=list(sw), seed_tolerance=seed_tolerance,
                            tolerance=tol, subset_order=subset_order, desc_dtype=desc_dtype, **mesh_kw)
        if not mesh_override and sol["stats"]["n_bad"] > 0:  # the quality gate's Err
            if f_index + 1 < g_index:
                f_index = g_index - 1
                pending = True
                if override:
                    mesh_override = True
                continue
            unsolvable = True
            break
        if mesh_override:
            if any(max(float(r["c_zncc"]), 0.0) < tolerance for r in sol["results"]):
                override_log.append(g_index)
            mesh_override = False
        if pending:
            if len(pairs) < n_pairs:
                reference_updates[len(pairs)] = True
            pending = False
        pairs.append(dict(f_index=f_index, g_index=g_index, sol=sol, seed_coord=tuple(seed_coord)))
        g_index += 1
        if g_index >= n_images:
            break
        if guide:
            disps = [[float(r["p"][0]), float(r["p"][1])] for r in sol["results"]]
            disp, new_warp = deformation_preconditioning(nodes, elements, disps, seed_coord, mesh_order, subset_order)
            seed_coord[0] += disp[0]
            seed_coord[1] += disp[1]
            n_copy = 6 * min(mesh_order, subset_order)
            sw = list(new_warp[:n_copy]) + [0.0] * (len(sw) - n_copy)
        if sequential:
            f_index = g_index - 1
            reference_updates[g_index - 1] = True
    return dict(pairs=pairs, override_log=override_log, reference_updates=reference_updates,
                all_converged=not unsolvable and g_index >= n_images, unsolvable=unsolvable)
