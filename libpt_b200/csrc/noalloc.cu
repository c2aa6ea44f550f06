// Allocation-free restricted (T) solve for small systems.
//
// Some callers cannot let a library call cudaMalloc: host programs that hand
// all device memory to their own pool allocator up front (a library-side
// cudaMalloc then fails, or silently breaks the program's memory
// accounting), and latency-sensitive loops in which cudaMalloc/cudaFree would
// synchronize the device and stall the program's other streams.  For them,
// libpt_rpt_dev_static runs the same engine as libpt_rpt_dev with every
// scratch buffer -- the padded operand copies, the contraction outputs of a
// batch of triples, the partial sums and the per-triple energies -- carved
// from the file-scope array below instead of allocated.  The caller passes
// the inputs (device pointers, pt.h layout) and receives the energy.
//
// The array is LIBPT_STATIC_SCRATCH_BYTES (64 MiB) of device memory that
// every GPU on which this file's device code is loaded keeps until the
// process exits.  Under CUDA's lazy module loading that happens at the first
// call on a device (the address lookup below loads it), so a caller whose
// pool allocator claims the device's memory makes one call -- any size that
// fits -- before creating its pool.  All calls share the array: each call
// clears the parts that must start at zero, later calls overwrite what
// earlier calls left, and two calls whose work overlaps on the GPU
// (different streams or threads at once) race on it and give wrong
// energies.  A call synchronizes the stream it is given (it reads whether
// f_ov is zero and the energies back), not the device.
#include <cuda_runtime.h>

#include <string>

#include "plan.h"
#include "pt.h"

#define LIBPT_API extern "C" __attribute__((visibility("default")))

static __device__ __align__(256) unsigned char
    g_static_scratch[LIBPT_STATIC_SCRATCH_BYTES];

namespace {

// Device address of the scratch array on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// with the device current.  It is looked up on every call (cheap once this
// file's device code is loaded) rather than cached: after a device reset the
// code is loaded again, possibly at another address.  The first lookup on a
// device loads this file's device code, which is when the array is reserved.
int scratch_address(void **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
  if (e != cudaSuccess || !p) {
    ptb::set_error(std::string("cudaGetSymbolAddress(static scratch): ") +
                   cudaGetErrorString(e));
    return LIBPT_ERR_CUDA;
  }
  *out = p;
  return LIBPT_OK;
}

}  // namespace

LIBPT_API int libpt_rpt_dev_static(size_t oa, size_t va, const double *d_ov,
                                   const double *f_ov, const double *t1,
                                   const double *t2, const double *i_oovo,
                                   const double *i_oovv,
                                   const double *i_ovvv, void *stream,
                                   double *e_out) {
  if (!e_out) {
    ptb::set_error("e_out is NULL");
    return LIBPT_ERR_ARG;
  }
  // size check first, from the sizes alone: a cheap lower bound (the padded
  // amplitude and OVVV copies), then the exact footprint of a plan whose
  // rounds hold one triple at least (sizing pass, no device work)
  const double lower = 8.0 * ((double)oa * oa * va * va * 2 +
                              (double)oa * va * va * va);
  const size_t need =
      (oa > 4096 || va > 4096 || lower > (double)LIBPT_STATIC_SCRATCH_BYTES)
          ? (size_t)lower
          : ptb::plan_footprint(0, oa, va, oa, va, 0, LIBPT_PREC_FP64, false, 1);
  // (a footprint of 0 means the sizing pass rejected the arguments)
  if (oa > 4096 || va > 4096 || need == 0 ||
      need > (size_t)LIBPT_STATIC_SCRATCH_BYTES) {
    ptb::set_error("libpt_rpt_dev_static: o=" + std::to_string(oa) +
                   ", v=" + std::to_string(va) + " needs " +
                   std::to_string(need) + " bytes of scratch; the static "
                   "scratch holds " +
                   std::to_string((size_t)LIBPT_STATIC_SCRATCH_BYTES) +
                   " (use libpt_rpt_dev for larger systems)");
    return LIBPT_ERR_ARG;
  }
  void *base = nullptr;
  if (int r = scratch_address(&base)) return r;
  const void *a[] = {d_ov, f_ov, t1, t2, i_oovo, i_oovv, i_ovvv};
  libpt_plan *p = nullptr;
  int r = ptb::plan_create(0, oa, va, oa, va, a, 0, LIBPT_PREC_FP64, false,
                           static_cast<cudaStream_t>(stream), &p, base,
                           (size_t)LIBPT_STATIC_SCRATCH_BYTES);
  if (!r) r = ptb::plan_run(p, nullptr, p->queue.size());
  if (!r) r = ptb::plan_energy(p, nullptr, 0, e_out);
  ptb::plan_destroy(p);
  return r;
}
