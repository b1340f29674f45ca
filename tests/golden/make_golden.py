"""Writes tests/golden/reference_kats.json and tests/golden/oracle_small.npz.

reference_kats.json -- the known-answer values of the reference crate's own
unit tests for this path, transcribed with their file:line (within the
geopyv-dev repository).  When $GPV_REFERENCE names a checkout of the
reference, every transcribed literal is looked up at its cited line, so a
mis-transcription fails loudly here; without it that check is skipped.

oracle_small.npz -- a small seeded synthetic pair (workload 1 at 1/8 scale)
with the FP64 oracle's coefficients and batch results, so tests can detect
an oracle change independently of the oracle itself.

    GPV_REFERENCE=<geopyv-dev checkout> python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("GPV_REFERENCE", "")

S2 = math.sqrt(2.0) / 4.0
KATS = [
    # convergence_norm (src/subset.rs:622-649)
    dict(name="norm_pure_translation", src="src/subset.rs:1427-1431", fn="norm",
         dp=[3.0, 4.0, 0.0, 0.0, 0.0, 0.0], size=1.0, expected=5.0, atol=1e-12, literal="vec![3.0, 4.0, 0.0, 0.0, 0.0, 0.0]"),
    dict(name="norm_zero", src="src/subset.rs:1435-1438", fn="norm", dp=[0.0] * 6, size=44.3, expected=0.0, atol=0.0,
         literal="convergence_norm(&dp, 44.3)"),
    dict(name="norm_gradient_term", src="src/subset.rs:1442-1448", fn="norm", dp=[0.0, 0.0, 2.0, 0.0, 0.0, 0.0],
         size=5.0, expected=10.0, atol=1e-12, literal="vec![0.0, 0.0, 2.0, 0.0, 0.0, 0.0]"),
    dict(name="norm_order0", src="src/subset.rs:1453-1456", fn="norm", dp=[0.3, 0.4], size=123.0, expected=0.5,
         atol=1e-12, literal="vec![0.3, 0.4]"),
    # zn_slice (src/subset.rs:698-704)
    dict(name="zn_slice_standardises", src="src/subset.rs:1461-1473", fn="zn_slice", x=[1.0, 2.0, 3.0],
         expected=[-1.0 / math.sqrt(2.0 / 3.0), 0.0, 1.0 / math.sqrt(2.0 / 3.0)], atol=1e-12, literal="[1.0, 2.0, 3.0]"),
    dict(name="zn_slice_zero_variance", src="src/subset.rs:1479-1486", fn="zn_slice", x=[5.0, 5.0, 5.0, 5.0],
         expected=[0.0, 0.0, 0.0, 0.0], atol=1e-6, literal="[5.0, 5.0, 5.0, 5.0]"),
    # eta_component (src/subset.rs:713-727)
    dict(name="eta_K3", src="src/subset.rs:1498-1510", fn="eta_component",
         modes=[[1.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0], [0.0, 0.0, 1.0]], grad_zn=[1.0, -1.0, 1.0, -1.0],
         e_centered=[1.0, 0.0, 0.0, 0.0], expected=S2, atol=1e-12, literal="std::f64::consts::SQRT_2 / 4.0"),
    dict(name="eta_K2", src="src/subset.rs:1522-1534", fn="eta_component",
         modes=[[1.0, 0.0], [-1.0, 0.0], [0.0, 1.0], [0.0, -1.0]], grad_zn=[1.0, -1.0, 1.0, -1.0],
         e_centered=[1.0, 0.0, 0.0, 0.0], expected=S2, atol=1e-12, literal="[-1.0, 0.0], // (ξ,ζ) = (-1, 0)"),
    dict(name="eta_K4", src="src/subset.rs:1555-1567", fn="eta_component",
         modes=[[1.0, 0.0, 0.0, 0.0], [-1.0, 0.0, 0.0, 0.0], [0.0, 0.0, 0.0, 1.0], [0.0, 0.0, 0.0, -1.0]],
         grad_zn=[1.0, -1.0, 1.0, -1.0], e_centered=[1.0, 0.0, 0.0, 0.0], expected=S2, atol=1e-12,
         literal="[0.0, 0.0, 0.0, -1.0], // (ξ,ζ) = (0, -1)"),
    dict(name="eta_non_negative", src="src/subset.rs:1538-1544", fn="eta_component",
         modes=[[1.0, 0.5, 0.2], [-0.3, 0.1, -0.7], [0.4, -0.4, 0.9]], grad_zn=[0.5, -1.2, 0.8],
         e_centered=[-0.6, 1.1, 0.2], expected=">=0", atol=0.0, literal="[[1.0, 0.5, 0.2], [-0.3, 0.1, -0.7], [0.4, -0.4, 0.9]]"),
    dict(name="eta_identical_images", src="src/subset.rs:1576-1600", fn="eta_identical",
         coord=[0.0, 0.0], f_coords=[[1.0, 0.0], [-1.0, 0.0], [0.0, 1.0], [0.0, -1.0]],
         grad_f=[[1.0, 0.5], [-1.0, 0.3], [0.2, 1.0], [-0.2, -1.0]], f=[10.0, 12.0, 9.0, 11.0], expected=0.0, atol=1e-10,
         literal="vec![10.0, 12.0, 9.0, 11.0]"),
    # znssd (src/subset.rs:654-669)
    dict(name="znssd_identical", src="src/subset.rs:1620-1626", fn="znssd_identical",
         f=[10.0, 50.0, 100.0, 200.0, 150.0], expected=0.0, atol=1e-12, literal="vec![10.0, 50.0, 100.0, 200.0, 150.0]"),
    dict(name="znssd_range", src="src/subset.rs:1630-1639", fn="znssd_range", f=[10.0, 50.0, 100.0, 200.0],
         g=[12.0, 48.0, 105.0, 190.0], expected=[0.0, 4.0], atol=0.0, literal="vec![12.0, 48.0, 105.0, 190.0]"),
    # compose_icgn (src/subset.rs:487-611)
    dict(name="compose_golden", src="src/subset.rs:1797-1810", fn="compose", p=[1.0, 0.5, 0.01, 0.02, -0.01, 0.005],
         dp=[0.1, 0.05, 0.001, 0.002, -0.001, 0.0005],
         expected=[0.89954843, 0.44797691, 0.00900896, 0.01797300, -0.00898650, 0.00451572], atol=1e-6,
         literal="0.89954843_f64, 0.44797691, 0.00900896, 0.01797300, -0.00898650, 0.00451572"),
    dict(name="compose_zero_delta", src="src/subset.rs:1703-1713", fn="compose", p=[1.0, 2.0, 0.1, 0.05, -0.1, 0.02],
         dp=[0.0] * 6, expected=[1.0, 2.0, 0.1, 0.05, -0.1, 0.02], atol=1e-10, literal="vec![1.0, 2.0, 0.1, 0.05, -0.1, 0.02]"),
    dict(name="compose_order0", src="src/subset.rs:1718-1725", fn="compose", p=[1.0, 2.0], dp=[0.5, 0.3],
         expected=[0.5, 1.7], atol=1e-12, literal="vec![0.5, 0.3]"),
    dict(name="compose_order0_zero", src="src/subset.rs:1729-1734", fn="compose", p=[1.5, -0.7], dp=[0.0, 0.0],
         expected=[1.5, -0.7], atol=1e-12, literal="vec![1.5, -0.7]"),
    dict(name="compose_pure_translation", src="src/subset.rs:1770-1779", fn="compose", p=[0.0] * 6,
         dp=[0.5, 0.3, 0.0, 0.0, 0.0, 0.0], expected=[-0.5, -0.3, 0.0, 0.0, 0.0, 0.0], atol=1e-10,
         literal="vec![0.5, 0.3, 0.0, 0.0, 0.0, 0.0]"),
    dict(name="compose_order2_length", src="src/subset.rs:1783-1788", fn="compose_len", p=[0.0] * 12,
         dp=[0.5, 0.3, 0.01, 0.01, 0.01, 0.01, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001], expected=12, atol=0.0,
         literal="vec![0.5, 0.3, 0.01, 0.01, 0.01, 0.01, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001]"),
    # warp convention suite (src/subset.rs:2211-2324, Q of src/particle.rs:2621)
    dict(name="warp_convention_Q", src="src/particle.rs:2621", fn="warp_convention",
         q=[0.1, -0.2, 0.02, 0.07, 0.03, -0.01, 0.004, 0.008, 0.005, 0.009, 0.006, -0.003],
         points=[[13.0, 7.0], [4.0, 15.0], [9.5, 9.5], [16.0, 2.0]], centre=[10.0, 10.0], expected=None, atol=1e-12,
         literal="[0.1, -0.2, 0.02, 0.07, 0.03, -0.01, 0.004, 0.008, 0.005, 0.009, 0.006, -0.003]"),
    dict(name="compose_order1_undoes_update", src="src/subset.rs:2272-2286", fn="compose_roundtrip1",
         dp=[0.05, -0.02, 0.004, -0.006, 0.003, 0.008], expected=None, atol=1e-12,
         literal="vec![0.05, -0.02, 0.004, -0.006, 0.003, 0.008]"),
    dict(name="compose_order2_third_order", src="src/subset.rs:2289-2305", fn="compose_roundtrip2",
         dp=[0.2, -0.1, 0.02, 0.05, -0.03, 0.01, 0.002, -0.001, 0.0015, 0.001, -0.002, 0.0012], expected=6.5, atol=0.0,
         literal="vec![0.2, -0.1, 0.02, 0.05, -0.03, 0.01, 0.002, -0.001, 0.0015, 0.001, -0.002, 0.0012]"),
    # masks (src/masks.rs:69-109, 199-263)
    dict(name="circle_5", src="src/masks.rs:275-296", fn="circle", radius=5, n_px=81, first=[0.0, -5.0], last=[0.0, 5.0],
         literal="assert_eq!(t.n_px, 81);"),
    dict(name="circle_25", src="src/subset.rs:1957", fn="circle", radius=25, n_px=1961, first=[0.0, -25.0],
         last=[0.0, 25.0], literal='assert_eq!(subset.n_px(), 1961, "n_px mismatch");'),
    dict(name="mask_update_zero", src="src/masks.rs:383-389", fn="mask_zero", literal="Array2::<u8>::zeros((20, 20))"),
    # B-spline (src/image.rs)
    dict(name="get_c_constant", src="src/image.rs:540-550", fn="get_c_constant", shape=[20, 25], border=5, value=77.0,
         rtol=1e-8, literal="Array2::from_elem((20, 25), val)"),
    dict(name="q_row_sums", src="src/image.rs:619-629", fn="q_row_sums", expected=[1.0, 0.0, 0.0, 0.0, 0.0, 0.0],
         atol=1e-15, literal="let expected = if r == 0 { 1.0 } else { 0.0 };"),
    dict(name="eval_matches_qcqt_blocks", src="src/image.rs:571-600", fn="qcqt_form", shape=[24, 28], border=6,
         points=[[3.25, 4.75], [10.0, 12.0], [0.0, 0.0], [15.999, 9.001], [7.5, 0.5], [26.3, 22.9]], atol=1e-11,
         literal="(3.25f64, 4.75f64), (10.0, 12.0), (0.0, 0.0), (15.999, 9.001), (7.5, 0.5), (26.3, 22.9)"),
    dict(name="grad_is_derivative", src="src/image.rs:635-647", fn="grad_fd", shape=[60, 60], border=8,
         points=[[30.0, 30.0], [30.25, 30.75], [30.5, 29.5], [31.9, 28.1]], atol=1e-4,
         literal="(30.0, 30.0), (30.25, 30.75), (30.5, 29.5), (31.9, 28.1)"),
    dict(name="constant_image_eval", src="src/subset.rs:1814-1821", fn="const_eval", shape=[4, 4], border=5,
         value=42.0, points=[[0.0, 0.0], [1.5, 2.25], [3.0, 3.0]], rtol=1e-8, literal="(0.0, 0.0), (1.5, 2.25), (3.0, 3.0)"),
    dict(name="far_out_of_range_clamp", src="src/subset.rs:1845-1868", fn="clamp", shape=[8, 9], border=5, atol=1e-3,
         literal="bspline_eval(1_000_000.0, 0.0, &img)"),
    # mesh propagation helpers (src/mesh.rs) -- checked against oracle/mesh_oracle.py
    dict(name="connectivity_order1_corner", src="src/mesh.rs:2657-2661", fn="mesh_connectivity",
         elements=[[0, 1, 2], [1, 3, 2]], order=1, idx=0, full=False, expected=[1, 2],
         literal="assert_eq!(result, vec![1, 2]);"),
    dict(name="connectivity_order1_shared_node", src="src/mesh.rs:2664-2668", fn="mesh_connectivity",
         elements=[[0, 1, 2], [1, 3, 2]], order=1, idx=1, full=False, expected=[0, 2, 3],
         literal="assert_eq!(result, vec![0, 2, 3]);"),
    dict(name="connectivity_order2_corner_gets_midpoints", src="src/mesh.rs:2671-2676", fn="mesh_connectivity",
         elements=[[0, 1, 2, 4, 5, 6], [1, 3, 2, 7, 8, 5]], order=2, idx=0, full=False, expected=[4, 6],
         literal="assert_eq!(result, vec![4, 6]);"),
    dict(name="connectivity_order2_midpoint_gets_corners", src="src/mesh.rs:2679-2684", fn="mesh_connectivity",
         elements=[[0, 1, 2, 4, 5, 6], [1, 3, 2, 7, 8, 5]], order=2, idx=4, full=False, expected=[0, 1],
         literal="assert_eq!(result, vec![0, 1]);"),
    dict(name="connectivity_indexed_matches", src="src/mesh.rs:2693-2720", fn="mesh_adjacency",
         cases=[[[[0, 1, 2], [1, 3, 2]], 1, 4], [[[0, 1, 2, 4, 5, 6], [1, 3, 2, 7, 8, 5]], 2, 9]],
         literal="let elements2 = array![[0usize, 1, 2, 4, 5, 6], [1, 3, 2, 7, 8, 5]];"),
    dict(name="find_seed_node_exact", src="src/mesh.rs:2724-2727", fn="mesh_seed",
         nodes=[[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]], coord=[1.0, 0.0], expected=1,
         literal="assert_eq!(find_seed_node(&nodes, [1.0, 0.0]), 1);"),
    dict(name="find_seed_node_nearest", src="src/mesh.rs:2730-2734", fn="mesh_seed",
         nodes=[[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]], coord=[0.4, 0.4], expected=0,
         literal="assert_eq!(find_seed_node(&nodes, [0.4, 0.4]), 0);"),
    dict(name="project_warp_second_order_terms", src="src/mesh.rs:2804-2813", fn="mesh_project",
         p={"4": 1.0, "8": 1.0}, dx=2.0, dy=3.0, slot=4, expected=3.0, atol=1e-12,
         literal="let p_proj = project_warp(&p, 2.0, 3.0);"),
    dict(name="project_warp_every_slot", src="src/mesh.rs:3237-3246", fn="mesh_project_quad",
         q=[0.1, -0.2, 0.02, 0.07, 0.03, -0.01, 0.004, 0.008, 0.005, 0.009, 0.006, -0.003], c=[2.0, -1.0],
         d=[3.0, 5.0], atol=1e-12, literal="let (cx, cy, dx, dy) = (2.0, -1.0, 3.0, 5.0);"),
    dict(name="affine_field_fit_recovers_exact_linear_field", src="src/mesh.rs:2819-2848", fn="mesh_affine_fit",
         nodes=[[0.0, 0.0], [10.0, 0.0], [0.0, 10.0], [10.0, 10.0], [5.0, 2.0]], u=[0.1, -0.05, 2.0],
         v=[-0.02, 0.08, -1.0], target=[3.0, 7.0], atol=1e-9, literal="v = -0.02*x + 0.08*y - 1.0"),
    dict(name="affine_field_fit_none_when_collinear", src="src/mesh.rs:2851-2857", fn="mesh_affine_collinear",
         nodes=[[0.0, 0.0], [1.0, 0.0], [2.0, 0.0]], target=[1.0, 5.0],
         literal="assert!(affine_field_fit(&nodes, [1.0, 5.0], &trusted, &p, 6).is_none());"),
    dict(name="precondition_warp_thresholds", src="src/mesh.rs:2861-2878", fn="mesh_precondition",
         nodes=[[0.0, 0.0], [1.0, 0.0]], c_zncc=[0.9, 0.95], p=[[1.0, 2.0, 0, 0, 0, 0], [3.0, 4.0, 0, 0, 0, 0]],
         target=[5.0, 5.0], atol=1e-12, literal="let one = precondition_warp(&nodes, [5.0, 5.0], &[1], &c_zncc, &p, 6);"),
]


def verify_provenance():
    if not REF or not os.path.isdir(REF):
        print("GPV_REFERENCE does not name a reference checkout; provenance not re-checked")
        return
    for k in KATS:
        path, lines = k["src"].split(":")
        a, _, b = lines.partition("-")
        a = int(a)
        b = int(b) if b else a
        text = open(os.path.join(REF, path), encoding="utf-8").read().splitlines()
        window = "\n".join(text[max(0, a - 3):b + 2])
        if k["literal"] not in window:
            raise SystemExit(f"{k['name']}: literal {k['literal']!r} not found at {k['src']}")
    print(f"provenance: {len(KATS)} literals found at their cited lines")


def write_oracle_fixture():
    sys.path[:0] = [os.path.join(ROOT, "geopyv-dev_b200"), os.path.join(ROOT, "oracle")]
    import numpy as np

    import oracle as O
    from gpv import synth
    O.build()
    W = synth.workload(1, scale_down=8)
    d = np.zeros(len(W["coords"]), O.DESC_DTYPE)
    d["coord"], d["radius"], d["order"] = W["coords"], 25, 1
    Cf = O.get_c(W["f"].astype(np.float64), 20)
    Cg = O.get_c(W["g"].astype(np.float64), 20)
    res = O.solve_batch(Cf, Cg, W["f"].shape, 20, d, max_norm=1e-5, max_iterations=15, eta=True)
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), f=W["f"], g=W["g"], desc=d.view(np.uint8),
                        result=res.view(np.uint8))
    print("oracle_small.npz:", len(d), "subsets")


if __name__ == "__main__":
    verify_provenance()
    with open(os.path.join(HERE, "reference_kats.json"), "w") as fh:
        json.dump(KATS, fh, indent=1)
    print("reference_kats.json:", len(KATS), "entries")
    write_oracle_fixture()
