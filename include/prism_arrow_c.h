/*
 * Arrow C Data Interface and C Device Data Interface structures.
 *
 * These are the ABI-stable structs defined by the Apache Arrow specification
 * ("The Arrow C data interface", "The Arrow C Device data interface"). The
 * layout must be bit-identical to every other producer/consumer, so the field
 * order and types below follow the published specification exactly; the
 * ARROW_C_DATA_INTERFACE / ARROW_C_DEVICE_DATA_INTERFACE guards let this file
 * coexist with any other copy of the same definitions.
 *
 * The reference operators exchange arrow-rs `RecordBatch`es and the reference
 * workspace already enables arrow's `ffi` feature (native/Cargo.toml:20;
 * native/prism-jni/src/lib.rs:9 imports FFI_ArrowArray / FFI_ArrowSchema), so
 * these structs are how a `RecordBatch` crosses the C ABI in prism_gpu.h.
 */
#ifndef PRISM_ARROW_C_H
#define PRISM_ARROW_C_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef ARROW_C_DATA_INTERFACE
#define ARROW_C_DATA_INTERFACE

#define ARROW_FLAG_DICTIONARY_ORDERED 1
#define ARROW_FLAG_NULLABLE 2
#define ARROW_FLAG_MAP_KEYS_SORTED 4

struct ArrowSchema {
  const char* format;
  const char* name;
  const char* metadata;
  int64_t flags;
  int64_t n_children;
  struct ArrowSchema** children;
  struct ArrowSchema* dictionary;
  void (*release)(struct ArrowSchema*);
  void* private_data;
};

struct ArrowArray {
  int64_t length;
  int64_t null_count;
  int64_t offset;
  int64_t n_buffers;
  int64_t n_children;
  const void** buffers;
  struct ArrowArray** children;
  struct ArrowArray* dictionary;
  void (*release)(struct ArrowArray*);
  void* private_data;
};

#endif /* ARROW_C_DATA_INTERFACE */

#ifndef ARROW_C_DEVICE_DATA_INTERFACE
#define ARROW_C_DEVICE_DATA_INTERFACE

typedef int32_t ArrowDeviceType;

#define ARROW_DEVICE_CPU 1
#define ARROW_DEVICE_CUDA 2
#define ARROW_DEVICE_CUDA_HOST 3
#define ARROW_DEVICE_CUDA_MANAGED 13

struct ArrowDeviceArray {
  struct ArrowArray array;
  int64_t device_id;
  ArrowDeviceType device_type;
  void* sync_event;
  int64_t reserved[3];
};

#endif /* ARROW_C_DEVICE_DATA_INTERFACE */

#ifdef __cplusplus
}
#endif

#endif /* PRISM_ARROW_C_H */
