// jit.hpp — per-query kernels generated at run time and compiled with NVRTC
// for sm_100a.
//
// The ahead-of-time kernels interpret a query's filter and expression
// programs node by node (eval.cuh); on a scan with few groups that
// interpretation costs thousands of instructions per row. The generator
// turns the same typed programs into straight-line CUDA C++ (column types and
// null-freedom fixed, literals in registers, 128-bit overflow checks only
// where the operand ranges need them) and instantiates the small-groups
// kernel body (agg_device.cuh) with it. Results are identical by
// construction: the generated code calls the same device helpers, in the
// same order of operations, as the interpreter.
#pragma once

#include <functional>
#include <string>

#include "runtime.hpp"

namespace prism {

struct Program;
struct AggArgs;

// False when PRISM_JIT=0 is set or NVRTC (libnvrtc.so.12) cannot be loaded;
// callers then launch the interpreting kernels.
bool jit_enabled();

// Kernel `name` of `source`, compiled once per process (cached by source
// text). A compile error is an engine bug: throws PRISM_ERR_INTERNAL with
// the compiler log.
const void* jit_get(const std::string& source, const char* name);

// Number of NVRTC compilations so far and their total wall time (ms).
void jit_stats(int64_t* compiles, double* ms);

// Source of the small-groups aggregation kernel `prism_tiny_agg` for the
// program `pg` over batch `b` (`a` holds the sources, ops and group columns;
// g groups, f64 = some Float64 SUM present). Empty when the program uses a
// construct the generator does not cover.
std::string jit_tiny_agg_source(const Program& pg, const Batch& b, const AggArgs& a, int g, bool f64);

// Source of the hashed-groups aggregation kernel `prism_hash_agg` (block
// size JoinKernelShape::hash_block, dynamic shared memory (2 + a.W) * 8 << a.ss_log2 bytes).
// With n_probe_cols >= 0, `b` is a joined batch (probe columns, then build
// columns) and the source is the fused join -> aggregate kernel
// `prism_join_agg` (join_body), reading build-side columns at the matched
// build row. Empty when the program uses a construct the generator does not
// cover.
constexpr int HASH_BLOCK_DEFAULT = 1024;
struct JoinKernelShape {
  int block = 512;      // threads per block
  int min_blocks = 3;   // blocks kept resident per SM (bounds registers and shared memory)
  int rows = 2;         // probe rows per thread in flight
  int hash_block = HASH_BLOCK_DEFAULT;  // threads per block of the hashed-groups kernel (no join)
};
std::string jit_hash_agg_source(const Program& pg, const Batch& b, const AggArgs& a, int n_probe_cols = -1,
                                const JoinKernelShape& join = JoinKernelShape{});

// The kernel `name` generated for this plan: the kernel made by `make` (a
// source generator over the same inputs) the first time a plan with this key
// is seen, the same kernel without generating its source again afterwards.
// The key holds everything the generators read: the program's host arrays,
// every column's type and attributes, the kernel arguments with each pointer
// reduced to null / non-null, and `extra` (the generator's own parameters).
// PRISM_JIT_PLAN_CACHE=0 generates the source every call.
const void* jit_plan_kernel(const Program& pg, const Batch& b, const AggArgs& a, const std::vector<int64_t>& extra,
                            const char* name, const std::function<std::string()>& make);

}  // namespace prism
