"""Compile-time limits of the CUDA kernels, parsed from the C header.

Like the reference's ``forcepho/kernel_limits.py:18-40``, which regex-parses
``kernel_limits.h``, the constants here are read from the one header the
kernels are compiled with (``include/forcepho_b200_limits.h``), so Python and
CUDA can never disagree on the struct sizes they imply.
"""

import os
import re

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "forcepho_b200_limits.h")

_define = re.compile(r"^\s*#define\s+(?P<name>[A-Z_][A-Z0-9_]*)\s+(?P<value>[-+0-9.eE]+)\s*$")


def _parse(path):
    macros = {}
    with open(path) as fp:
        for line in fp:
            m = _define.match(line)
            if m:
                v = m.group("value")
                try:
                    macros[m.group("name")] = int(v)
                except ValueError:
                    macros[m.group("name")] = float(v)
    return macros


macros = _parse(HEADER)
MAXBANDS = macros["MAXBANDS"]
MAXSOURCES = macros["MAXSOURCES"]
NPARAMS = macros["NPARAMS"]
MAX_EXP_ARG = macros["MAX_EXP_ARG"]
MAXRADII = macros["MAXRADII"]

__all__ = ["MAXBANDS", "MAXSOURCES", "NPARAMS", "MAX_EXP_ARG", "MAXRADII", "macros"]
