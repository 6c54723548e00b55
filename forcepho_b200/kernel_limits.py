"""Compile-time limits shared with the CUDA library.

The first five are the reference's (forcepho/src/kernel_limits.h:5-26, exposed
in python by forcepho/kernel_limits.py); they fix the byte layout of the
``Source`` and ``Response`` structs and so are part of the ABI.  The last two
are limits of this implementation, which lifts the reference's 30-source and
48 KB-per-band caps.
"""

MAXBANDS = 30
MAXSOURCES = 30
NPARAMS = 7
MAX_EXP_ARG = 36.0
MAXRADII = 10

MAX_ACTIVE_SOURCES = 1024
MAX_PSF_PER_SOURCE = 1024

__all__ = ["MAXBANDS", "MAXSOURCES", "NPARAMS", "MAX_EXP_ARG", "MAXRADII",
           "MAX_ACTIVE_SOURCES", "MAX_PSF_PER_SOURCE"]
