"""Reading the reference's WRF input files (mgpu.cu:343-417).

The reference loads six text files of one value per line (`%lf`), each a field-major
array [nfield][48][20][48] with i fastest: wrfchem.txt (82 fields), wrfmoist.txt (6),
wrfph.txt (28), wrfphy.txt (3), wrfrad.txt (29) and wrfvdrog3.txt (17, not used by the
chemistry).  The files themselves are not shipped with the reference.  `load_text_fields`
reads such a directory into the arrays `Solver.convert_wrf` takes; `save_text_fields`
writes the same format (used by the round-trip test and to hand synthetic fields to the
reference's own reader).

Parsing text costs seconds per time level (3.8 M values in wrfchem.txt alone).  The binary
form keeps the same arrays as raw little-endian float64 files (`wrfchem.bin`, ...) with a
small header of the field count and dimensions; `load_binary_fields` maps them without
parsing (`mmap=True`) or reads them in one call, and `text_to_binary` converts a directory
once.
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


# Binary form: 16-byte header "RADM2WRF" + 4 x int32 (nfield, nj, nk, ni), then the
# [nfield][nj][nk][ni] float64 array, little-endian, i fastest (the text files' order).
_MAGIC = b"RADM2WRF"
_HEADER = 8 + 4 * 4


def _bin_name(name):
    return os.path.splitext(name)[0] + ".bin"


def save_binary_fields(fields, directory):
    os.makedirs(directory, exist_ok=True)
    for k, (name, nfield) in FILES.items():
        a = np.ascontiguousarray(fields[k], dtype="<f8")
        if a.ndim != 4 or a.shape[0] != nfield:
            raise ValueError("%s: expected [%d][nj][nk][ni], got %s" % (k, nfield, a.shape))
        with open(os.path.join(directory, _bin_name(name)), "wb") as f:
            f.write(_MAGIC)
            f.write(np.asarray(a.shape, dtype="<i4").tobytes())
            f.write(a.tobytes())


def _read_bin(path, nfield, mmap):
    with open(path, "rb") as f:
        head = f.read(_HEADER)
    if len(head) != _HEADER or head[:8] != _MAGIC:
        raise ValueError("%s: not a RADM2WRF binary field file" % path)
    shape = tuple(int(v) for v in np.frombuffer(head[8:], dtype="<i4"))
    if shape[0] != nfield or min(shape) <= 0:
        raise ValueError("%s: header %s, expected %d fields" % (path, shape, nfield))
    count = int(np.prod(shape))
    size = os.path.getsize(path) - _HEADER
    if size != count * 8:
        raise ValueError("%s: %d data bytes, header says %d" % (path, size, count * 8))
    if mmap:
        return np.memmap(path, dtype="<f8", mode="r", offset=_HEADER, shape=shape)
    return np.fromfile(path, dtype="<f8", count=count, offset=_HEADER).reshape(shape)


def load_binary_fields(directory, mmap=False):
    """The arrays of `load_text_fields` from the binary form (read-only maps with mmap=True)."""
    return {k: _read_bin(os.path.join(directory, _bin_name(name)), n, mmap) for k, (name, n) in FILES.items()}


def text_to_binary(src_directory, dst_directory, dims=DIMS):
    """Convert the reference's text files once; later runs load the binary form."""
    save_binary_fields(load_text_fields(src_directory, dims), dst_directory)
