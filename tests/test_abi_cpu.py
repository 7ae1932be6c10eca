"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes as C
import os
import re

import pytest

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
    assert L.hdb_set_join_tiles(None, 1) == _lib.HDB_ERR_ARG
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
    assert C.sizeof(_lib.Graph) == 56


def test_ctypes_structs_match_the_c_header(tmp_path):
    """Every struct the ctypes binding declares has the size and field
    offsets the C compiler gives include/hdb/hdb.h."""
    import shutil
    import subprocess
    from gpu_hdbscan_b200 import _lib
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    pairs = {"hdb_knn_params": _lib.KnnParams, "hdb_params": _lib.Params, "hdb_graph": _lib.Graph,
             "hdb_run_stats": _lib.RunStats, "hdb_instance": _lib.Instance}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "hdb/hdb.h"', "int main(void) {"]
    for cname, cls in pairs.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "sizes.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "sizes"
    inc = os.path.join(ROOT, "include")
    subprocess.run(["gcc", "-I", inc, "-o", str(exe), str(src)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())
    for cname, cls in pairs.items():
        assert int(got[cname]) == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, (cname, fname)
