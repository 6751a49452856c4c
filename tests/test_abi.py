"""The C-ABI library loads and exports exactly what include/orf_b200.h declares (no GPU needed)."""
import subprocess

from open_rendering_framework_b200 import _native as nat


def test_library_loads_and_reports_version():
    L = nat.lib()
    assert L.pt_version() >= 100
    assert L.pt_last_error_message() is not None


def test_every_declared_function_is_exported_and_bound():
    declared = nat.declared_functions()
    assert declared, "no declarations found in include/orf_b200.h"
    out = subprocess.run(["nm", "-D", "--defined-only", nat.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [f for f in declared if f not in exported]
    assert not missing, "declared but not exported: %s" % missing
    unbound = [f for f in declared if f not in nat.SIGNATURES]
    assert not unbound, "declared but missing from the Python binding: %s" % unbound
    stale = [f for f in nat.SIGNATURES if f not in declared]
    assert not stale, "bound in Python but not declared in the header: %s" % stale


def test_invalid_arguments_are_rejected_without_a_gpu():
    L = nat.lib()
    # null pointers and a bad enum are caught on the host before any device work
    assert L.pt_bsdf_queries(None, None, 16, 0, 8, 0.66, None, None, None, None, None) == 1
    assert L.pt_rng_streams(7, None, 4, 4, None, None) == 1
    assert b"kind" in L.pt_last_error_message()
