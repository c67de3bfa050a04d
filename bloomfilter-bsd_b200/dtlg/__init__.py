"""dtlg -- B200-native build/probe of the DTL filter family (blocked Bloom,
sectorized, zoned, cuckoo, blocked cuckoo and classic Bloom filters) behind
the reference's filter API.

The hot path is libdtlg.so (sm_100a kernels behind the C ABI in
include/dtlg.h); this package is the host-side mirror of the reference's
filter_base / filter interface over it.
"""
from ._lib import DtlgError, InvalidConfig, SizeError, lib  # noqa: F401
from .filter import (MAGIC, POWER_OF_TWO, bbf_32, bbf_64, bcf, blocked_bloomfilter_config,  # noqa: F401
                     bloomfilter_logic, cf, construct, cuckoofilter_config, filter, filter_base, probe_t, zbbf_32,
                     zbbf_64)

__all__ = [
    "DtlgError", "InvalidConfig", "SizeError", "lib", "MAGIC", "POWER_OF_TWO", "bbf_32", "bbf_64", "bcf", "bloomfilter_logic",
    "blocked_bloomfilter_config", "cf", "construct", "cuckoofilter_config", "filter", "filter_base",
    "probe_t", "zbbf_32", "zbbf_64",
]
