"""Regenerate the golden fixtures under tests/golden/ from the reference tree.

Run in a container where the reference is mounted (its path is the first
argument, default /root/reference).  It copies the reference's own 380-byte
unit-test geometry (src/unittests/resources/four_cube.gmy), its iolet fixtures
(iolet.txt, config_file_inlet.xml, velocity_inlet.txt,
config_file_velocity_inlet.xml, config_new_velocity_inlets.xml), the table of
J0(i^(3/2) x) that its Bessel unit test holds (bessel_j0_table.json, parsed
from src/unittests/util/BesselTests.h), and records, for the
geometries shipped with the reference's example cases, the site counts and
table checksums that the oracle reads from them.
"""

import hashlib
import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
CASES = ["cases/pipe/pipe.gmy", "cases/bifurcation/bifurcation_lores/bifurcation.gmy",
         "cases/FiveExit/SixBranch.gmy", "cases/UnevenArms/UnevenArms.gmy", "cases/elasticWallsExample/pipe.gmy"]


def sha(a):
    return hashlib.sha256(a.tobytes()).hexdigest()


def main():
    src = os.path.join(REF, "src/unittests/resources/four_cube.gmy")
    shutil.copyfile(src, os.path.join(HERE, "four_cube.gmy"))
    # The file-pressure iolet fixtures of InOutLetTests::TestFileConstruct
    # (src/unittests/lbtests/iolets/InOutLetTests.h:117-162).
    # The velocity iolet fixtures of InOutLetTests::TestWomersleyVelocityConstruct and
    # TestFileVelocityConstruct (InOutLetTests.h:200-332).
    for name in ("iolet.txt", "config_file_inlet.xml", "velocity_inlet.txt", "config_file_velocity_inlet.xml",
                 "config_new_velocity_inlets.xml"):
        shutil.copyfile(os.path.join(REF, "src/unittests/resources", name), os.path.join(HERE, name))
    # BesselTests::TestUsedRange (src/unittests/util/BesselTests.h): J0(i^(3/2) x) for
    # x = 0, 0.1, ..., 20, compared there at an absolute 1e-6.
    text = open(os.path.join(REF, "src/unittests/util/BesselTests.h")).read()
    table = text[text.index("mathematica[] = {"):]
    table = table[:table.index("};")]
    vals = [(float(a), float(b)) for a, b in re.findall(r"Complex\(\s*([-+0-9.eE]+)\s*,\s*([-+0-9.eE]+)\s*\)", table)]
    assert len(vals) == 201
    with open(os.path.join(HERE, "bessel_j0_table.json"), "w") as fh:
        json.dump({"x": [k / 10.0 for k in range(201)], "j0": vals, "abs_tol": 1e-6}, fh)
    out = {}
    for rel in CASES:
        lat = O.Lattice(os.path.join(REF, rel))
        w, io, t, i = lat.sitedata()
        out[rel] = {"sites": lat.n, "type_counts": lat.type_counts().tolist(),
                    "sha256_neighbours": sha(lat.neighbours()), "sha256_coords": sha(lat.coords()),
                    "sha256_wall_mask": sha(w), "sha256_iolet_mask": sha(io)}
    with open(os.path.join(HERE, "reference_geometries.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()
