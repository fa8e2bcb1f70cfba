"""B200-native (sm_100a) CSR SpGEMM with the method and interface of
geektrove/GPUSpGEMM's ``proposal`` path.

Host side of the library: ``.csr`` I/O, seeded synthetic inputs, and a Python
mirror of the reference interface over the C ABI of ``libspgemm_b200.so``.
"""
from .csr import HostCSR, load_csr, reference_equal, save_csr  # noqa: F401

__all__ = ["HostCSR", "load_csr", "save_csr", "reference_equal", "DeviceCSR", "Handle",
           "proposal", "proposal_host", "get_nip", "SpgemmError"]


def __getattr__(name):
    # the native binding loads lazily so that the pure-host parts import
    # without the built library
    if name in ("DeviceCSR", "Handle", "proposal", "proposal_host", "get_nip",
                "default_handle"):
        from . import api
        return getattr(api, name)
    if name == "SpgemmError":
        from ._native import SpgemmError
        return SpgemmError
    raise AttributeError(name)
