"""Loads the committed golden fixtures (tests/golden/*.npz) into engine inputs."""
import os

import numpy as np

from forte_b200 import integrals as I

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(k: int):
    """Returns (ints, na, nb, irrep, multiplicity, reference energy) for integrals-fcidump-k."""
    z = np.load(os.path.join(HERE, f"fcidump{k}.npz"))
    src = z if "values" in z else np.load(os.path.join(HERE, f"fcidump{int(z['integrals_from'])}.npz"))
    d = I.fcidump_from_entries(str(z["header"]), src["values"], src["index"])
    ints, na, nb, irrep, mult = I.active_space_from_fcidump(
        d, z["frozen_docc"], z["restricted_docc"], z["active"], int(z["nel"]), int(z["multiplicity"]))
    return ints, na, nb, irrep, mult, float(z["reffci"])
