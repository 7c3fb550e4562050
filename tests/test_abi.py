"""C ABI checks that need no GPU: the library loads, exports every function
include/prism_gpu.h declares, and the ctypes mirror matches the C layouts."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

import prism_gpu
from prism_gpu import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "prism_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(prism_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(prism_gpu.LIB_PATH):
        import __graft_entry__

        __graft_entry__.build()
    return prism_gpu.lib()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_no_device_error(lib):
    assert b"sm_100a" in lib.prism_version()
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        with pytest.raises(prism_gpu.PrismError) as e:
            prism_gpu.Context()
        assert e.value.kind == "Cuda"


def test_null_arguments_return_status_not_abort(lib):
    h = C.c_void_p()
    assert lib.prism_ctx_create(0, 0, None) == 3  # InvalidArgument
    # every operator rejects a null context instead of crashing
    assert lib.prism_hash_join(None, None, None, None, C.byref(h)) == 3
    assert lib.prism_hash_aggregate(None, None, None, C.byref(h)) == 3
    assert lib.prism_batch_num_rows(None) == -1


STRUCTS = {
    "prism_join_config": _abi.prism_join_config,
    "prism_agg_expr": _abi.prism_agg_expr,
    "prism_agg_config": _abi.prism_agg_config,
    "prism_scalar": _abi.prism_scalar,
    "prism_pred_node": _abi.prism_pred_node,
    "prism_predicate": _abi.prism_predicate,
    "prism_expr_node": _abi.prism_expr_node,
    "prism_expr_clause": _abi.prism_expr_clause,
    "prism_expr": _abi.prism_expr,
    "struct ArrowArray": _abi.ArrowArray,
    "struct ArrowSchema": _abi.ArrowSchema,
    "struct ArrowDeviceArray": _abi.ArrowDeviceArray,
}


def test_ctypes_layouts_match_the_header():
    src = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        src.append(f'printf("%s %zu\\n", "{cname}", sizeof({cname}));')
        for fname, _ in py._fields_:
            src.append(f'printf("%s.%s %zu\\n", "{cname}", "{fname}", offsetof({cname}, {fname}));')
    src.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(c, "w").write("\n".join(src))
        subprocess.run(["gcc", c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.strip().splitlines())
    for cname, py in STRUCTS.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)
