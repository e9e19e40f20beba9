// Device -> pageable host copies at PCIe speed.
//
// A D2H copy into ordinary (pageable, possibly never touched) host memory
// runs at a few GB/s, and pinning a 100 GB result array costs seconds.  The
// copier instead moves rows through a ring of pinned buffers on its own copy
// stream, and a pool of host threads moves each landed buffer into the
// destination in parallel (taking the destination's first-touch page faults
// in parallel too), overlapping both with the GPU's compute.  A destination
// that is page-locked already (gsmc_host_alloc's result buffers, or any
// cudaHostAlloc'd / registered memory) is written by the DMA directly.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace gsmc {

class HostCopier {
 public:
  // The copier of the current device (created on first use).
  static HostCopier* for_current_device();

  // Copy `rows` rows of `width` bytes from device memory (src, row pitch
  // spitch) to host memory (dst, row pitch dpitch) once `ready` has completed
  // on the device.  Returns after enqueueing; a cudaError_t.
  int enqueue(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
              size_t rows, cudaEvent_t ready);

  // Record on the copy stream an event that completes when every D2H copy
  // enqueued so far has finished reading device memory.
  int record_reads_done(cudaEvent_t ev);

  // Block until every enqueued copy is in host memory; returns the first
  // error seen since the last drain (cudaSuccess if none).
  int drain();

  ~HostCopier();

 private:
  HostCopier();
  struct Impl;
  Impl* impl_;
};

}  // namespace gsmc
