// rb_internal.h -- definitions shared by the library's translation units (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace rb {

// message returned by rb_last_error() on the calling thread
extern thread_local std::string g_error;

// counts one kernel launch (rb_launch_count)
void note_launch();

// device-wide exclusive scan of int32 counts on `st`: data[0..n) -> exclusive prefix sums, data[n] = total,
// *total_out = total (when not null).  n = min(*n_dev, n_host) with a device count, else n_host.
// `partial` needs kScanPartials int32 of scratch.
constexpr int kScanGrid = 592;   // blocks of each scan pass (4 x 148 SMs)
constexpr int kScanPartials = kScanGrid + 1;
void scan(int32_t* data, const int32_t* n_dev, int n_host, int32_t* partial, int32_t* total_out, cudaStream_t st);

}  // namespace rb
