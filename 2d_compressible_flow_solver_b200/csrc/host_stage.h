// Copies between a caller's pageable host array and device memory through a
// pinned staging buffer, in chunks: host threads copy each chunk into (or out
// of) the staging buffer while the DMA engine moves the chunk before (after)
// it.  A pageable cudaMemcpyAsync is staged by the driver one small buffer at a
// time, about 11 GB/s on a B200 host for a 537 MB state; this pipeline runs
// near the pinned copy's PCIe rate.  The bytes are copied unchanged, so the
// result is the same bit for bit as the plain copy.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace cfs {

// Whether `p` is ordinary pageable host memory (not page-locked, not device
// or managed memory): only such arrays take the staged copies.
bool host_is_pageable(const void* p);

// Smallest copy worth the pipeline (smaller ones go through cudaMemcpyAsync).
constexpr size_t kStagedCopyMinBytes = size_t(32) << 20;

// Host -> device: `bytes` of `src` (pageable) to `dst` on `stream`, through
// `stage` (pinned, >= bytes).  Returns when every copy is enqueued; the
// staging buffer is in use until the stream reaches them.
cudaError_t upload_staged(void* dst, const void* src, size_t bytes, void* stage, cudaStream_t stream, int device);

// Device -> host: `bytes` of `src` to `dst` (pageable) after the work already
// on `stream`, through `stage`.  Returns when `dst` holds the data.
cudaError_t download_staged(void* dst, const void* src, size_t bytes, void* stage, cudaStream_t stream, int device);

}  // namespace cfs
