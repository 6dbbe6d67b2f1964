"""CPU checks of the C-ABI boundary: the library loads and exports every symbol the headers declare.

No compute call is made here (there is no GPU in this container); argument
validation that needs no device is exercised through the Python mirror.
"""
import ctypes
import glob
import os
import re

import pytest

from conftest import PKG, ROOT

DECL = re.compile(r"^\s*(?:cudaError_t|void|int|uint32_t|uint64_t|size_t|bool|const char\s*\*|bc_\w+\s*\*?)\s+\**(bc_\w+)\s*\(",
                  re.M)


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names.update(DECL.findall(open(h).read()))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_symbols()
    for required in ("bc_ntt_context_create", "bc_ntt_context_destroy", "bc_batch_ntt_internal",
                     "bc_batch_ntt_out_of_place", "bc_batch_ntt_in_place"):
        assert required in names


def test_library_exports_every_declared_symbol():
    path = os.path.join(PKG, "libbc_ntt.so")
    if not os.path.exists(path):
        pytest.fail(f"{path} not built (run __graft_entry__.build())")
    L = ctypes.CDLL(path)
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_mirror_binds_every_symbol():
    import bc_ntt

    assert set(bc_ntt.SIGNATURES) <= set(declared_symbols())
    bc_ntt.lib()  # loads and declares without touching a device
