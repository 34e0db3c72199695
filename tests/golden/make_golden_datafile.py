"""Regenerate the golden ARTS data file from the reference's own writer.

Drives ``oracle/_ref/libref_fileio.so`` -- the reference's library/fileio_c.c, compiled
unchanged by ``oracle/f90_to_c.py`` -- in the call order of tools/init_flow/param.f90:113-148
(param_write_data) on a seeded 5 x 4 x 3 grid of 4 variables, and stores the file as
``tests/golden/data_ref_small.bin``. It pins the library's data-file reader where the reference
tree is absent.

    python oracle/f90_to_c.py <reference>/combustion && python tests/golden/make_golden_datafile.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import RefFileIO  # noqa: E402

NAMES = ["RHO", "T", "H2O", "ZMIX"]


def fields():
    rng = np.random.default_rng(2026)
    return np.asfortranarray(rng.standard_normal((5, 4, 3, len(NAMES))))


def main():
    RefFileIO().write_data(os.path.join(HERE, "data_ref_small.bin"), fields(), NAMES, dt=2.5e-6, time=0.125)


if __name__ == "__main__":
    main()
