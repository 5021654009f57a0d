"""qcmaquis_b200: B200-native two-site DMRG effective-Hamiltonian path.

Python host layer over the C-ABI in include/qcm_b200.h (libqcm_b200.so, built
in-tree).  Import fails if the native library is missing; there is no CPU
fallback for the device path.
"""
from ._lib import lib as _native, QcmError  # noqa: F401


def version() -> str:
    return _native.qcm_version().decode()
