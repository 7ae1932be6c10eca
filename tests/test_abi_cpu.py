"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes as C
import os
import re

from conftest import ROOT


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "hdb", "hdb.h")).read()
    return sorted(set(re.findall(r"HDB_API\s+[\w\s\*]+?\b(hdb_\w+)\s*\(", src)))


def test_header_declares_the_python_export_list():
    from gpu_hdbscan_b200 import _lib
    assert declared_symbols() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(libpath):
    lib = C.CDLL(libpath)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_version_and_last_error_without_gpu(libpath):
    from gpu_hdbscan_b200 import _lib
    L = _lib.load(libpath)
    assert L.hdb_version().decode().startswith("hdb_b200")
    assert isinstance(L.hdb_last_error(), bytes)


def test_null_context_is_an_argument_error(libpath):
    from gpu_hdbscan_b200 import _lib
    L = _lib.load(libpath)
    assert L.hdb_set_stream(None, None) == _lib.HDB_ERR_ARG
    assert b"NULL" in L.hdb_last_error()
    assert L.hdb_destroy(None) == _lib.HDB_OK


def test_struct_layouts_match_reference_records():
    from gpu_hdbscan_b200 import _lib
    # NNDElement 8 B, MSTedge 12 B, SingleLinkageNode / CondensedTreeNode 16 B
    from oracle import oracle as O
    assert O.MST_EDGE.itemsize == 12
    assert O.LINKAGE_NODE.itemsize == 16
    assert O.CONDENSED_NODE.itemsize == 16
    assert O.STABILITY.itemsize == 8
    assert C.sizeof(_lib.KnnParams) == 16
    assert C.sizeof(_lib.Params) == 32
    assert C.sizeof(_lib.Graph) == 56
