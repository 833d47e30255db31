"""Generates the committed golden fixtures from the reference itself.

Runs the reference's own code (oracle/_ref/libbbrt_ref.so, built by
oracle/build_ref.sh from the reference's headers) on seeded synthetic scenes
and stores its outputs, so tests can pin the oracle port and the GPU path
against the reference on machines where the reference sources are absent.

    python tests/golden/make_golden.py

Fixtures (numpy .npz, kept small by storing only bouncing rays' hits and a
seeded sample of escaped rays' end points):
  triangles.npz        tests/Triangle_Intersect.cpp's four triangles and rays
  two_spheres.npz      16384-ray plane source, coarse n = 9, tol 1e-12, <= 20 bounces
  two_spheres_ref_constants.npz   same scene, the reference's own constants
                       (n = 100, tol 1e-3), first 2048 rays
  tetra_spheres.npz    first 4096 rays of the seeded 10-degree cone source
  ellipsoids.npz       first 2048 rays of the seeded 20-degree cone source
  plane_counts.npz     PlaneSourceDriver hit counts on the two-sphere scene
  bounce_map.npz       BounceMapDriver max bounces / error counts on it
"""
from __future__ import annotations

import hashlib
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from billardballraytracing3d_b200 import scenes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
K = 4


def scene_digest(patches) -> str:
    h = hashlib.sha256()
    for p in patches:
        h.update(np.array([p.imax, p.jmax, p.zone_id], dtype=np.int64).tobytes())
        for f in ("u_nodes", "v_nodes") + scenes.Patch.FIELDS:
            h.update(np.ascontiguousarray(getattr(p, f), dtype="<f8").tobytes())
    return h.hexdigest()


def array_digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype="<f8").tobytes())
    return h.hexdigest()


def ray_digest(o, d) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(o, dtype="<f8").tobytes())
    h.update(np.ascontiguousarray(d, dtype="<f8").tobytes())
    return h.hexdigest()


def trace_fixture(name, n_rays, coarse_n=None, tol=None, n_escaped_sample=512):
    patches, o, d, maxb, cn, tl = scenes.workload(name, n_rays)
    cn = coarse_n or cn
    tl = tol or tl
    with tempfile.TemporaryDirectory() as tmp:
        ref = oracle.Reference.from_patches(patches, tmpdir=tmp, coarse_n=cn, newton_tol=tl)
        r = ref.trace(o, d, maxb, K=K, nthreads=os.cpu_count())
        zones = np.array([ref_zone for ref_zone in (oracle.Reference.lib().ref_zone_id(ref.h, k)
                                                    for k in range(ref.n_objects))], dtype=np.int64)
        diag, msag = ref.scene_diagonal, ref.max_patch_sagitta
        setup = [ref.patch_setup(k) for k in (0, len(patches) // 2, len(patches) - 1)]
        ref.close()
    bounced = np.nonzero(r["bounce_count"] > 0)[0]
    rng = np.random.Generator(np.random.PCG64(7))
    esc = np.nonzero(r["status"] == 0)[0]
    esc_sample = np.sort(rng.choice(esc, size=min(n_escaped_sample, esc.size), replace=False))
    fx = dict(
        scene_sha256=scene_digest(patches), ray_sha256=ray_digest(o, d),
        n_rays=np.int64(o.shape[0]), max_bounces=np.int64(maxb), coarse_n=np.int64(cn), newton_tol=np.float64(tl),
        scene_diagonal=np.float64(diag), max_patch_sagitta=np.float64(msag), zone_ids=zones,
        status=r["status"].astype(np.int8), bounce_count=r["bounce_count"].astype(np.int16),
        err_zone=r["err_zone"],
        bounced=bounced.astype(np.int32), hit_object=r["hit_object"][bounced].astype(np.int32),
        hit_point=r["hit_point"][bounced], bounced_end_point=r["end_point"][bounced],
        escaped_sample=esc_sample.astype(np.int32), escaped_end_point=r["end_point"][esc_sample],
        escaped_exit_dir=r["exit_dir"][esc_sample],
        setup_index=np.array([0, len(patches) // 2, len(patches) - 1], dtype=np.int32),
        setup_box=np.stack([s["box"] for s in setup]), setup_centroid=np.stack([s["centroid"] for s in setup]),
        setup_max_sagitta=np.array([s["max_sagitta"] for s in setup]),
        # coarse grids as digests (the n = 100 grids would be megabytes)
        setup_coarse_sha256=np.array([array_digest(s["coarse_xyz"], s["sagitta"], s["cell_normal"]) for s in setup]),
        cpu_seconds=np.float64(r["seconds"]), cpu_threads=np.int64(os.cpu_count()),
    )
    return fx


def main():
    if not oracle.reference_available():
        raise SystemExit("oracle/_ref/libbbrt_ref.so is missing: run oracle/build_ref.sh first")

    # tests/Triangle_Intersect.cpp:18-31: four triangles, BVH leaf_threshold 1, four rays
    tris = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0], [10, 0, 0, 11, 0, 0, 10, 1, 0],
                     [0, 0, 5, 1, 0, 5, 0, 1, 5], [-5, 0, 0, -4, 0, 0, -5, 1, 0]], dtype=np.float64)
    ro = np.array([[0.2, 0.2, -1], [10.2, 0.2, -1], [100, 100, -1], [0.2, 0.2, 10]], dtype=np.float64)
    rd = np.array([[0, 0, 1], [0, 0, 1], [0, 0, 1], [0, 0, -1]], dtype=np.float64)
    bt, bo, ft, fo = oracle.Reference.triangle_queries(tris, 1, ro, rd)
    np.savez_compressed(os.path.join(OUT, "triangles.npz"), tris=tris, origins=ro, dirs=rd,
                        bvh_t=bt, bvh_obj=bo, brute_t=ft, brute_hit=fo)

    np.savez_compressed(os.path.join(OUT, "two_spheres.npz"), **trace_fixture("two_spheres", None))
    np.savez_compressed(os.path.join(OUT, "two_spheres_ref_constants.npz"),
                        **trace_fixture("two_spheres", 2048, coarse_n=100, tol=1e-3, n_escaped_sample=128))
    np.savez_compressed(os.path.join(OUT, "tetra_spheres.npz"), **trace_fixture("tetra_spheres", 4096))
    np.savez_compressed(os.path.join(OUT, "ellipsoids.npz"), **trace_fixture("ellipsoids", 2048))

    patches = scenes.scene_two_spheres()
    with tempfile.TemporaryDirectory() as tmp:
        scenes.write_scene_dir(tmp, patches)
        oracle.Reference.lib().ref_set_constants(9, 20, 1e-12)
        ref = oracle.Reference(tmp, coarse_n=9, newton_tol=1e-12)
        c0, c1, dd = (-3.0, -3.0, 4.0), (3.0, 3.0, 4.0), (0.3, 0.0, -1.0)
        counts, _ = ref.plane_source(c0, c1, dd, 64, 48, 20, False, nthreads=os.cpu_count())
        counts_direct, _ = ref.plane_source(c0, c1, dd, 64, 48, 20, True, nthreads=os.cpu_count())
        ref.close()
        np.savez_compressed(os.path.join(OUT, "plane_counts.npz"), corner0=np.array(c0), corner1=np.array(c1),
                            direction=np.array(dd), nx=np.int64(64), ny=np.int64(48), max_bounces=np.int64(20),
                            counts=counts, counts_direct=counts_direct, scene_sha256=scene_digest(patches))
        # BounceMapDriver samples "<dir><prefix><i>.txt" by 1-based index: patches 1..8,
        # half of the first sphere's +x face, which looks at the second sphere
        sample_dir = os.path.join(tmp, "bm") + os.sep
        os.makedirs(sample_dir)
        for k, p in enumerate(patches):
            scenes.write_patch_file(os.path.join(sample_dir, f"p{k + 1}.txt"), p)
        first, last = 1, 8
        mb, er, _ = oracle.Reference.bounce_map(sample_dir, "p", first, last, 3, 4, 6, 120.0, 20,
                                                nthreads=os.cpu_count())
        np.savez_compressed(os.path.join(OUT, "bounce_map.npz"), first=np.int64(first), last=np.int64(last),
                            grid_n=np.int64(3), theta_n=np.int64(4), phi_n=np.int64(6), cone=np.float64(120.0),
                            max_bounces=np.int64(20), max_b=mb, errors=er, scene_sha256=scene_digest(patches))
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
