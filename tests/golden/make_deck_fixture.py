"""Copies the reference's shipped input deck (hopp3d.inp: twelve numeric
lines, the poured packing of 10,000 spheres the reference runs) into
tests/golden/, so that the GPU tests can run it where the reference checkout
is absent.

    DEM_REFERENCE_DIR=<reference checkout> python tests/golden/make_deck_fixture.py
"""
import os
import pathlib

HERE = pathlib.Path(__file__).resolve().parent


def main():
    src = pathlib.Path(os.environ.get("DEM_REFERENCE_DIR", "/root/reference")) / "hopp3d.inp"
    deck = src.read_text().splitlines()[:12]
    assert all(ln.split() for ln in deck), "expected twelve numeric lines"
    (HERE / "hopp3d.inp").write_text("\n".join(deck) + "\n")
    print(f"wrote {HERE / 'hopp3d.inp'} from {src}")


if __name__ == "__main__":
    main()
