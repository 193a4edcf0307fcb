"""Regenerate the golden fixtures in tests/golden/ from the reference.

Run where the reference tree exists, with the oracle built against it:

  make -C oracle REF=<reference root>
  python tests/golden/make_golden.py <reference root>

(or set RQ_REFERENCE instead of the argument).  The GPU box never needs the
reference: the tests read only the files this script writes.

  exp0_ray_stats.json   published SW BVH4 statistics, results/exp0_ray_stats.csv
  radv_layouts.json     compute_tree_layout (include/radv_bvh.hpp:193-215)
  ref_terrain1000.npz   createTessellatedTerrain(1000) and the reference's
                        SoftwareBVH / SoftwareBVH4 bytes for it
  ref_dynamic_grids.npz generate_dynamic_grid_mesh(N, 1.25) for the builder
                        verification sizes N = 64, 256, 1024, 4096
  radv_dumps.json       dump_bvh_structure text of those grids' RADV images
  ref_median_soups.npz  the reference's SoftwareBVH / SoftwareBVH4 bytes for
                        random soups without repeated centroid values
"""
import csv
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as O  # noqa: E402

def reference_root():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RQ_REFERENCE")
    if not ref or not os.path.isfile(os.path.join(ref, "common", "software_bvh.hpp")):
        sys.exit("usage: make_golden.py <reference root>  (or RQ_REFERENCE=<reference root>)")
    return ref


def main():
    REF = reference_root()
    rows = []
    with open(os.path.join(REF, "results", "exp0_ray_stats.csv")) as f:
        for r in csv.DictReader(f):
            if r["HitRate_SW_pct"] == "N/A":
                continue
            rows.append(dict(tris=int(r["Triangles"]), pattern=r["RayPattern"],
                             hw_hit_pct=float(r["HitRate_HW_pct"]), sw_hit_pct=float(r["HitRate_SW_pct"]),
                             box_tests=float(r["AvgBoxTests_PerRay"]), tri_tests=float(r["AvgTriTests_PerRay"])))
    with open(os.path.join(HERE, "exp0_ray_stats.json"), "w") as f:
        json.dump({"source": "results/exp0_ray_stats.csv", "rays": 1048576, "camera": [0, 50, -45],
                   "look_at": [0, 0, 5], "rows": rows}, f, indent=1)

    lay = {}
    for n in (1, 3, 4, 5, 16, 17, 64, 256, 1024, 4096, 4097, 65536, 100000):
        lay[str(n)] = O.ref_tree_layout(n)
    with open(os.path.join(HERE, "radv_layouts.json"), "w") as f:
        json.dump(lay, f, indent=1)

    pos, idx = O.ref_terrain(1000)
    n2, tris, n4 = O.ref_build(pos, idx)
    np.savez_compressed(os.path.join(HERE, "ref_terrain1000.npz"), pos=pos, idx=idx, nodes2=n2.view(np.uint8),
                        tris=tris.view(np.uint8), nodes4=n4.view(np.uint8))

    grids = {}
    for n in (64, 256, 1024, 4096):
        tri9, cen = O.ref_dynamic_grid(n, 1.25)
        grids[f"tri9_{n}"] = tri9
        grids[f"cen_{n}"] = cen
    np.savez_compressed(os.path.join(HERE, "ref_dynamic_grids.npz"), **grids)

    # the reference decoder's text (dump_bvh_structure) of the RADV images of
    # those grids (images from the fast-builder restatement, byte-equal to
    # the device builder's)
    dumps = {}
    for n in (64, 256, 1024, 4096):
        img = O.radv_build(grids[f"tri9_{n}"])
        dumps[str(n)] = O.ref_dump_bvh_structure(img.tobytes())
    with open(os.path.join(HERE, "radv_dumps.json"), "w") as f:
        json.dump(dumps, f, indent=1)

    # median-split trees of soups whose float32 centroids never repeat a
    # value on an axis (the soup of tests/conftest.py, repeats removed)
    med = {}
    for tag, n, seed, leaf in (("a", 3000, 11, 4), ("b", 8000, 12, 2)):
        rng = np.random.default_rng(seed)
        c = rng.uniform(-1.0, 1.0, size=(n, 1, 3)).astype(np.float32)
        e = rng.uniform(-0.05, 0.05, size=(n, 3, 3)).astype(np.float32)
        v = (c + e).astype(np.float32)
        cen = ((v[:, 0] + v[:, 1]) + v[:, 2]) / np.float32(3.0)
        keep = np.ones(n, bool)
        for a in range(3):
            _, inv, cnt = np.unique(cen[:, a], return_inverse=True, return_counts=True)
            keep &= cnt[inv] == 1
        pos = np.ascontiguousarray(v[keep].reshape(-1, 3))
        n2, tris, n4 = O.ref_build(pos, np.arange(len(pos), dtype=np.uint32), leaf)
        med.update({f"pos_{tag}": pos, f"leaf_{tag}": np.uint32(leaf), f"nodes2_{tag}": n2.view(np.uint8),
                    f"tris_{tag}": tris.view(np.uint8), f"nodes4_{tag}": n4.view(np.uint8)})
    np.savez_compressed(os.path.join(HERE, "ref_median_soups.npz"), **med)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
