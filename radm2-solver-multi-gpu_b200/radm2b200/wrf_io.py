"""Reading the reference's WRF input files (mgpu.cu:343-417).

The reference loads six text files of one value per line (`%lf`), each a field-major
array [nfield][48][20][48] with i fastest: wrfchem.txt (82 fields), wrfmoist.txt (6),
wrfph.txt (28), wrfphy.txt (3), wrfrad.txt (29) and wrfvdrog3.txt (17, not used by the
chemistry).  The files themselves are not shipped with the reference.  `load_text_fields`
reads such a directory into the arrays `Solver.convert_wrf` takes; `save_text_fields`
writes the same format (used by the round-trip test and to hand synthetic fields to the
reference's own reader).
"""
import os

import numpy as np

FILES = {"chem": ("wrfchem.txt", 82), "moist": ("wrfmoist.txt", 6), "ph": ("wrfph.txt", 28),
         "phy": ("wrfphy.txt", 3), "rad": ("wrfrad.txt", 29)}
DIMS = (48, 20, 48)  # nj, nk, ni


def _read(path, nfield, dims):
    vals = np.loadtxt(path, dtype=np.float64, ndmin=1)
    need = nfield * int(np.prod(dims))
    if vals.size < need:
        raise ValueError("%s: %d values, need %d" % (path, vals.size, need))
    return vals[:need].reshape((nfield,) + tuple(dims))


def load_text_fields(directory, dims=DIMS):
    """dict ph/chem/rad/phy/moist of [nfield][nj][nk][ni] arrays from the reference's files."""
    return {k: _read(os.path.join(directory, name), n, dims) for k, (name, n) in FILES.items()}


def save_text_fields(fields, directory):
    os.makedirs(directory, exist_ok=True)
    for k, (name, _) in FILES.items():
        np.savetxt(os.path.join(directory, name), np.asarray(fields[k]).ravel(), fmt="%.17g")
