"""Pack the reference-kernel golden vectors into tests/golden/ref_kernels.npz.

The vectors come from oracle/_ref/ref_golden, which runs the reference's own
neiglist.cu kernels (calcHashD, findCellStartD, addTwoArraysD,
updatepositionD, vprojec, vscale, and the bookkeeping of calculateforceiwD /
calculateforcepairD with no-contact stand-ins for the absent force laws) on a
GPU and writes raw binaries plus manifest.txt:

    make -C oracle ref                       # here, from the reference sources
    oracle/_ref/ref_golden <outdir>          # on a GPU
    python tests/golden/make_ref_golden.py <outdir>
"""
import pathlib
import sys

import numpy as np

DT = {"f8": np.float64, "u4": np.uint32}


def main(src):
    src = pathlib.Path(src)
    arrays = {}
    for line in (src / "manifest.txt").read_text().split("\n"):
        if not line.strip():
            continue
        name, dt, count = line.split()
        a = np.fromfile(src / f"{name}.bin", dtype=DT[dt])
        assert a.size == int(count), name
        arrays[name] = a
    out = pathlib.Path(__file__).resolve().parent / "ref_kernels.npz"
    np.savez_compressed(out, **arrays)
    print(f"wrote {out} ({out.stat().st_size} bytes, {len(arrays)} arrays)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_ref_golden.py <directory written by oracle/_ref/ref_golden>")
    main(sys.argv[1])
