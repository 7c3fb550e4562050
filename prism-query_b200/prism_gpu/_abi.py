"""ctypes mirror of include/prism_arrow_c.h and include/prism_gpu.h.

Struct layouts here must match the C headers field for field; the
``test_abi`` tests compare sizes and offsets against the compiled library.
"""
from __future__ import annotations

import ctypes as C

import pyarrow as pa

# ----------------------------------------------------------- Arrow C ABI ----


class ArrowSchema(C.Structure):
    pass


ArrowSchema._fields_ = [
    ("format", C.c_char_p),
    ("name", C.c_char_p),
    ("metadata", C.c_char_p),
    ("flags", C.c_int64),
    ("n_children", C.c_int64),
    ("children", C.POINTER(C.POINTER(ArrowSchema))),
    ("dictionary", C.POINTER(ArrowSchema)),
    ("release", C.CFUNCTYPE(None, C.POINTER(ArrowSchema))),
    ("private_data", C.c_void_p),
]


class ArrowArray(C.Structure):
    pass


ArrowArray._fields_ = [
    ("length", C.c_int64),
    ("null_count", C.c_int64),
    ("offset", C.c_int64),
    ("n_buffers", C.c_int64),
    ("n_children", C.c_int64),
    ("buffers", C.POINTER(C.c_void_p)),
    ("children", C.POINTER(C.POINTER(ArrowArray))),
    ("dictionary", C.POINTER(ArrowArray)),
    ("release", C.CFUNCTYPE(None, C.POINTER(ArrowArray))),
    ("private_data", C.c_void_p),
]


class ArrowDeviceArray(C.Structure):
    _fields_ = [
        ("array", ArrowArray),
        ("device_id", C.c_int64),
        ("device_type", C.c_int32),
        ("sync_event", C.c_void_p),
        ("reserved", C.c_int64 * 3),
    ]


ARROW_DEVICE_CPU = 1
ARROW_DEVICE_CUDA = 2
ARROW_DEVICE_CUDA_HOST = 3


class ExportedBatch:
    """A pyarrow RecordBatch exported through the C Data Interface.

    The C structs are borrowed by the callee; ``release()`` (or garbage
    collection) gives the buffers back to pyarrow.
    """

    def __init__(self, batch: pa.RecordBatch):
        self.batch = batch
        self.array = ArrowArray()
        self.schema = ArrowSchema()
        batch._export_to_c(C.addressof(self.array), C.addressof(self.schema))

    @property
    def array_ptr(self):
        return C.pointer(self.array)

    @property
    def schema_ptr(self):
        return C.pointer(self.schema)

    def release(self):
        if self.array.release:
            self.array.release(C.pointer(self.array))
        if self.schema.release:
            self.schema.release(C.pointer(self.schema))

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class ExportedSchema:
    """A pyarrow Schema exported through the C Data Interface (as a struct)."""

    def __init__(self, schema: pa.Schema):
        self.schema = ArrowSchema()
        schema._export_to_c(C.addressof(self.schema))

    @property
    def schema_ptr(self):
        return C.pointer(self.schema)

    def __del__(self):
        try:
            if self.schema.release:
                self.schema.release(C.pointer(self.schema))
        except Exception:
            pass


def import_batch(array: ArrowArray, schema: ArrowSchema) -> pa.RecordBatch:
    """Moves an exported struct array (callee-produced) into pyarrow."""
    return pa.RecordBatch._import_from_c(C.addressof(array), C.addressof(schema))


# ------------------------------------------------------------ prism ABI ----

PRISM_OK = 0
ERROR_NAMES = {
    1: "Arrow",
    2: "SchemaMismatch",
    3: "InvalidArgument",
    4: "Execution",
    5: "Join",
    6: "UnsupportedAggregation",
    7: "Internal",
    8: "TableFull",
    9: "NoMemory",
    10: "Timeout",
    11: "Cuda",
}


class prism_join_config(C.Structure):
    _fields_ = [
        ("join_type", C.c_int32),
        ("n_keys", C.c_int32),
        ("probe_keys", C.POINTER(C.c_int32)),
        ("build_keys", C.POINTER(C.c_int32)),
    ]


class prism_agg_expr(C.Structure):
    _fields_ = [("column", C.c_int32), ("func", C.c_int32), ("output_name", C.c_char_p)]


class prism_parquet_scan_config(C.Structure):
    _fields_ = [
        ("uris", C.POINTER(C.c_char_p)),
        ("n_uris", C.c_int32),
        ("predicate", C.c_void_p),
        ("projection", C.POINTER(C.c_int32)),
        ("n_projection", C.c_int32),
        ("batch_size", C.c_int64),
        ("skip_expand", C.c_int32),
        ("target_schema", C.c_void_p),
    ]


class prism_parquet_scan_stats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("files", "row_groups", "row_groups_skipped", "pages", "compressed_bytes",
                                          "inflated_bytes", "decoded_bytes")]


class prism_sort_key(C.Structure):
    _fields_ = [("column", C.c_int32), ("descending", C.c_int32), ("nulls_first", C.c_int32)]


class prism_agg_config(C.Structure):
    _fields_ = [
        ("n_group_by", C.c_int32),
        ("group_by", C.POINTER(C.c_int32)),
        ("n_aggs", C.c_int32),
        ("aggs", C.POINTER(prism_agg_expr)),
    ]


class prism_scalar(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("reserved", C.c_int32),
        ("i64", C.c_int64),
        ("f64", C.c_double),
        ("str", C.c_char_p),
        ("str_len", C.c_int64),
    ]


class prism_pred_node(C.Structure):
    _fields_ = [("op", C.c_int32), ("column", C.c_int32), ("value", prism_scalar)]


class prism_predicate(C.Structure):
    _fields_ = [("nodes", C.POINTER(prism_pred_node)), ("n_nodes", C.c_int32)]


class prism_expr_node(C.Structure):
    _fields_ = [
        ("op", C.c_int32),
        ("column", C.c_int32),
        ("literal", prism_scalar),
        ("n_clauses", C.c_int32),
        ("has_else", C.c_int32),
        ("clause_begin", C.c_int32),
        ("reserved", C.c_int32),
    ]


class prism_expr_clause(C.Structure):
    _fields_ = [("pred_begin", C.c_int32), ("pred_len", C.c_int32)]


class prism_expr(C.Structure):
    _fields_ = [
        ("nodes", C.POINTER(prism_expr_node)),
        ("n_nodes", C.c_int32),
        ("preds", C.POINTER(prism_pred_node)),
        ("n_preds", C.c_int32),
        ("clauses", C.POINTER(prism_expr_clause)),
        ("n_clauses", C.c_int32),
    ]


def int_array(values):
    values = list(values)
    arr = (C.c_int32 * max(1, len(values)))(*values)
    return arr


TUNE_MAX = 16


class TuneResult(C.Structure):
    """prism_tune_result (include/prism_gpu.h)."""

    _fields_ = [("n_candidates", C.c_int32), ("best", C.c_int32), ("ms", C.c_double * TUNE_MAX),
                ("desc", (C.c_char * 64) * TUNE_MAX)]

    def as_dict(self):
        cands = [{"settings": self.desc[i].value.decode(), "ms": self.ms[i]} for i in range(self.n_candidates)]
        return {"candidates": cands, "best": cands[self.best] if cands else None}
