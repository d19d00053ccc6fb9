"""thirring -- host-side mirror of the thirring-rhmc fermion-path routines on B200.

The functions of `Lattice` carry the names and argument meanings of the
reference's Fortran routines (dirac.F90 dslash/dslashd, gauge.F90 coef,
measure_module.F90 congrad, qmrherm_module.F90 qmrherm, derivs_module.F90
derivs, gaussian.F90 gauss0/gaussp, ...) and operate on numpy arrays in the
reference's Fortran layout.  All compute runs in libthirring_b200.so on the
GPU; errors are raised as ThirringError with the library's status code.
"""
from ._lib import LibraryMissing, header_functions, lib  # noqa: F401
from .api import (CON_MPIIO, CON_SERIAL, EVEN_ODD, FP32_REF, FP64, MIXED_BF16, MIXED_FP32, NATURAL,  # noqa: F401
                  SHAMIR, WILSON, Lattice, Pack, ThirringError, TrajResult, field3, links, ps_field, read_con,
                  read_remez_file, readseed, remez_set, saveseed, shift_out, spinor, write_con, zolo_coeffs)
