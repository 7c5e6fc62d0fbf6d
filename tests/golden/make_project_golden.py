"""Golden projections from the reference's own emdata::project3d (src/EMReader/emdata.cpp:
891-996), run through oracle/_ref/ref_project (built by oracle/ref_project.sh from the
reference sources; host code only).  Inputs are bit-reproducible (fixture_data), so the
fixtures hold only the projections.

    python tests/golden/make_project_golden.py      # writes tests/golden/project_<case>.npz
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
from fixture_data import PROJECTION_CASES, bump_volume  # noqa: E402

HARNESS = os.path.join(REPO, "oracle", "_ref", "ref_project")


def write_mrc(path: str, vol: np.ndarray):
    nz, ny, nx = vol.shape
    hdr = np.zeros(256, dtype="<i4")
    hdr[0], hdr[1], hdr[2], hdr[3] = nx, ny, nz, 2
    with open(path, "wb") as fh:
        fh.write(hdr.tobytes())
        fh.write(np.ascontiguousarray(vol, dtype="<f4").tobytes())


def main():
    if not os.path.exists(HARNESS):
        subprocess.run(["bash", os.path.join(REPO, "oracle", "ref_project.sh")], check=True)
    for name, (size, blobs, seed, ri, angles) in PROJECTION_CASES.items():
        vol = bump_volume(size, blobs, seed)
        with tempfile.TemporaryDirectory() as d:
            write_mrc(os.path.join(d, "v.mrc"), vol)
            with open(os.path.join(d, "a.txt"), "w") as fh:
                fh.write("".join(f"{a!r} {b!r} {c!r}\n" for a, b, c in angles))
            subprocess.run([HARNESS, os.path.join(d, "v.mrc"), str(ri), os.path.join(d, "a.txt"),
                            os.path.join(d, "p.raw")], check=True, capture_output=True)
            proj = np.fromfile(os.path.join(d, "p.raw"), dtype="<f4").reshape(len(angles), size, size)
        np.savez_compressed(os.path.join(HERE, f"project_{name}.npz"), projections=proj,
                            volume_sum=np.float64(vol.astype(np.float64).sum()))
        print(name, proj.shape, float(np.abs(proj).max()))


if __name__ == "__main__":
    main()
