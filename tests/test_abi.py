"""The C-ABI library loads and exports every function include/gpart_b200.h
declares (no compute call is made here)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "gpart_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gp_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_api():
    names = declared_functions()
    for required in ("gp_partition", "gp_partition_device", "gp_context_create", "gp_verify", "gp_read_csr_int64"):
        assert required in names


def test_library_exports_every_declared_symbol(gp):
    lib = gp.library()
    missing = [name for name in declared_functions() if not hasattr(lib, name)]
    assert not missing, missing


def test_version_and_error_strings(gp):
    assert "sm_100a" in gp.version()
    assert isinstance(gp.library().gp_last_error(), bytes)


def test_product_does_not_load_the_oracle(gp):
    """The product library links no oracle code: its dynamic dependencies
    and exported symbols contain nothing from oracle/."""
    lib = gp.library()
    assert not hasattr(lib, "orc_partition")
    src = open(os.path.join(ROOT, "acc-gp_b200", "__init__.py")).read()
    assert "oracle" not in src.lower()
