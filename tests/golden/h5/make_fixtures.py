"""Copies the HDF5 files the reference's own storage layer wrote (H5Cpp, default properties) into
this directory as golden fixtures for thor_b200/h5.py, and records their SHA-256 in MANIFEST.

    python tests/golden/h5/make_fixtures.py /path/to/reference
    THOR_REFERENCE_DIR=/path/to/reference python tests/golden/h5/make_fixtures.py

The files are data, written by the reference's bin/esp for three configurations (an Earth
Held-Suarez run at glevel 4 / 32 levels, a deep hot-Jupiter set-up and an Earth set-up at
glevel 5 / 20 levels); the tests read them and pin their contents.
"""
import hashlib
import os
import shutil
import sys

SOURCES = {
    "planet_earth_hs_g4L32.h5": "ifile/esp_initial_planet.h5",
    "planet_deep_g4L40.h5": "ic_special/gen_ic_deep/esp_initial_planet.h5",
    "planet_earth_g5L20.h5": "ic_special/gen_ic_earth/esp_initial_planet.h5",
}


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    lines = []
    for name, rel in SOURCES.items():
        dst = os.path.join(here, name)
        shutil.copyfile(os.path.join(ref, rel), dst)
        with open(dst, "rb") as f:
            lines.append("%s  %s  (from %s)" % (hashlib.sha256(f.read()).hexdigest(), name, rel))
    with open(os.path.join(here, "MANIFEST"), "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("THOR_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: make_fixtures.py REFERENCE_DIR (or set THOR_REFERENCE_DIR)")
    main(ref)
