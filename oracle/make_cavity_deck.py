"""Write a short copy of the reference's lid-driven-cavity example
(exemplos/lid_driven_cavity.zip of the reference checkout: 64,000
hexahedra, SIMPLE with Rhie-Chow, WALE LES, second-order upwind) for the
end-to-end drop-in test: three SIMPLE iterations per time step, a cell and
node print every step in ASCII VTK.  Test infrastructure only.

    python oracle/make_cavity_deck.py <reference checkout> <output dir>
"""
from __future__ import annotations

import os
import shutil
import sys
import tempfile
import zipfile


def main(ref: str, out: str) -> int:
    src = os.path.join(ref, "exemplos", "lid_driven_cavity.zip")
    with tempfile.TemporaryDirectory() as tmp:
        zipfile.ZipFile(src).extractall(tmp)
        case = os.path.join(tmp, "lid_driven_cavity")
        simple = os.path.join(case, "config", "simple.dat")
        text = open(simple).read()
        open(simple, "w").write(text.replace("maxIt        5000", "maxIt        3"))
        deck = os.path.join(case, "cavidadeQH2.dat")
        text = open(deck).read()
        text = text.replace("transient config: BACKWARD 0.05e0 0.5e+00 static",
                            "transient config: BACKWARD 0.05e0 0.05e+00 static")
        text = text.replace("setPrint time 0.1 binary node cell vel pres eddyViscosity end",
                            "setPrint time 0.05 node cell vel pres end")
        open(deck, "w").write(text)
        if os.path.isdir(out):
            shutil.rmtree(out)
        shutil.copytree(case, out)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1], sys.argv[2]))
