"""Generates tests/golden/driver_errors.txt from the reference itself.

Compiles tests/cpp/driver_errors.cpp (which uses only the reference's public
API) against the reference's own headers, with oracle/shim standing in for
MKL and MPI, runs it on the driver test scene and keeps its output: the
exception type and text of every bad-argument and misuse case.  The same
program compiled against the C++ mirror headers must print the same lines.

    python tests/golden/make_driver_errors.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from billardballraytracing3d_b200 import scenes  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "driver_errors.txt")
SAMPLE_PREFIX = "samples/s"


def driver_scene():
    """Two unit spheres, 96 patches each on 5x5 nodes."""
    return scenes.scene_two_spheres()


def write_driver_scene(directory: str, n_samples: int = 2):
    """The scene as one file per patch in `directory`, plus copies of its
    first n_samples patches as <directory>/samples/s<i>.txt (1-based) for
    BounceMapDriver.  Returns the patch list."""
    patches = driver_scene()
    scenes.write_scene_dir(directory, patches)
    os.makedirs(os.path.join(directory, "samples"), exist_ok=True)
    for i in range(n_samples):
        scenes.write_patch_file(os.path.join(directory, "samples", f"s{i + 1}.txt"), patches[i])
    return patches


def main(ref_root: str | None = None) -> None:
    import oracle
    ref_root = ref_root or oracle.reference_root()
    tmp = tempfile.mkdtemp(prefix="driver_errors_")
    try:
        exe = os.path.join(tmp, "driver_errors")
        subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-I", os.path.join(ROOT, "oracle", "shim"),
                        "-I", os.path.join(ref_root, "include"), os.path.join(ROOT, "tests", "cpp", "driver_errors.cpp"),
                        "-o", exe], check=True)
        scene = os.path.join(tmp, "scene") + "/"
        write_driver_scene(scene)
        out = subprocess.run([exe, scene, SAMPLE_PREFIX], check=True, capture_output=True, text=True).stdout
        with open(OUT, "w") as f:
            f.write(out)
        print(out, end="")
    finally:
        shutil.rmtree(tmp)


if __name__ == "__main__":
    main(*sys.argv[1:])
