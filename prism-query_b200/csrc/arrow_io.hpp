// arrow_io.hpp — Arrow C Data Interface <-> device batches.
#pragma once

#include "runtime.hpp"

namespace prism {

// Imports a struct array; host buffers are copied to the device, device
// buffers (device_buffers = true) are wrapped without a copy.
Batch import_batch(Ctx& ctx, const ArrowArray* a, const ArrowSchema* s, bool device_buffers);
Batch import_device_batch(Ctx& ctx, const ArrowDeviceArray* a, const ArrowSchema* s);
// Copies a device batch into freshly allocated host buffers (caller releases).
void export_batch(Ctx& ctx, const Batch& b, ArrowArray* a, ArrowSchema* s);

// A fixed-width, null-free host output column filled by asynchronous
// device-to-host copies: `values` is page-locked pool memory (or malloc'd
// when pinning fails) of at least the requested bytes; `meta` carries the
// type, name, nullability and decimal precision / scale (no device buffers).
struct HostOutCol {
  ColP meta;
  void* values = nullptr;
  std::shared_ptr<void> hold;
};
HostOutCol host_out_column(ColP meta, size_t bytes);
// A host struct array described without copying: per child, its metadata
// (type, name, nullability, precision / scale) in `meta`, and for a
// fixed-width child its host values pointer at the array's first row.
struct HostView {
  ColP meta;
  const void* values = nullptr;
  int64_t null_count = 0;
};
std::vector<HostView> host_view(const ArrowArray* a, const ArrowSchema* s);
// A host struct array of `rows` rows over the columns' buffers (released
// back to the pool by the consumer's release callback).
void export_host_columns(const std::vector<HostOutCol>& cols, int64_t rows, ArrowArray* a, ArrowSchema* s);

// The engine type of an Arrow format string (TY_*; decimal precision /
// scale for "d:p,s"); false when unsupported.
bool arrow_format_type(const char* format, int32_t& type, int32_t& precision, int32_t& scale);

// A host struct array as a Batch whose column pointers are HOST pointers
// (no copy; bitmaps not starting on a byte boundary are realigned into
// `keep`). For host-side code only (the packed exchange format on the host).
Batch host_batch(const ArrowArray* a, const ArrowSchema* s, std::vector<std::shared_ptr<std::vector<uint8_t>>>& keep);
// Exports a Batch of HOST pointers (kept alive by `hold`) as a struct array.
void export_host_batch(const Batch& b, const std::shared_ptr<void>& hold, ArrowArray* a, ArrowSchema* s);

// Page-locked host staging from the process-wide recycling pool: a buffer of
// at least `bytes` (its size in *size), or nullptr when pinning fails.
void* pinned_get(size_t bytes, size_t* size);
void pinned_put(void* p, size_t size);

}  // namespace prism
