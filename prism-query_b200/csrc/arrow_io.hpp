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

// Page-locked host staging from the process-wide recycling pool: a buffer of
// at least `bytes` (its size in *size), or nullptr when pinning fails.
void* pinned_get(size_t bytes, size_t* size);
void pinned_put(void* p, size_t size);

}  // namespace prism
