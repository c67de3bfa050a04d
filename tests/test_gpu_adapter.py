"""The C++ drop-in: bloomfilter-bsd_b200/adapter/gpu_filter.hpp, a subclass of
the reference's own dtl::filter::filter_base, driven by virtual calls through
a filter_base* (tests/adapter/filter_base_known_answer.cpp): the reference's
known answer (filter_test.cpp:16-40), member probes of sectorized, zoned and
cuckoo filters, single-key calls, size(), name(), and the reference's
exception for an invalid config.  The driver is compiled against the
reference's header by build() (make -C tests/adapter)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "tests", "adapter", "_build", "filter_base_known_answer")


def test_filter_base_adapter_known_answer():
    if not os.path.exists(DRIVER):
        pytest.skip("the adapter's driver is not built (needs the reference tree at build time)")
    r = subprocess.run([DRIVER], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")
