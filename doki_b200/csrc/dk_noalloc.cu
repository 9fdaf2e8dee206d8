/*
 * Allocation-free marginals: dk_marginals_noalloc (include/dokigpu.h).
 *
 * Some callers cannot let a library allocate device memory: frameworks that
 * own every device byte through their own allocator (a caching allocator, a
 * fixed arena sized to an HBM budget), and latency-critical loops where a
 * cudaMalloc / cudaFree would synchronise the device.  This entry point runs
 * the same one-sweep marginal reduction as dk_marginals on an amplitude array
 * the caller owns, writing into an output array the caller owns, and takes its
 * per-block scratch from the file-scope array below instead of allocating it.
 *
 * The array lives in every device that loads this library, for as long as
 * the process runs.  All calls share it and it keeps the last call's
 * contents; each reduction block overwrites every slot the final pass reads,
 * so nothing needs clearing between calls.  Calls that overlap on the device
 * (different streams, or other threads without ordering) race on the array.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "dk_internal.h"
#include "dk_kernels.h"

namespace {

/* Per-block partial sums: up to kNoallocBlocks blocks x kPartialStride
 * doubles (256 x 64 x 8 bytes = 128 KiB per device). */
constexpr int kNoallocBlocks = 256;
static __device__ __align__(256) double g_noalloc_partials[kNoallocBlocks * dk::kPartialStride];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_addr[kMaxDevices] = { nullptr };

} // namespace

extern "C" int dk_marginals_noalloc(const void *amps, unsigned num_qubits, int precision,
				    double *out, void *stream)
{
	DK_TRACE();
	if (!amps || !out || (precision != DK_C64 && precision != DK_C128) || num_qubits == 0)
		return DK_ERR_ARG;
	if (num_qubits > DK_NOALLOC_MAX_QUBITS)
		return DK_ERR_NOALLOC_LIMIT;
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
		cudaGetLastError();
		return DK_ERR_NODEV;
	}
	double *scratch = nullptr;
	{
		/* set-up, once per device, with that device current: the host-side
		 * symbol is not a device address, so ask the runtime for it */
		std::lock_guard<std::mutex> lk(g_noalloc_mu);
		if (!g_noalloc_addr[dev]) {
			void *p = nullptr;
			if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) {
				cudaGetLastError();
				return DK_ERR_CUDA;
			}
			g_noalloc_addr[dev] = static_cast<double *>(p);
		}
		scratch = g_noalloc_addr[dev];
	}
	dk::Scratch s;
	s.partials = scratch;
	s.u64 = nullptr;
	s.marg = out;
	cudaError_t e = dk::launch_marginals_blocks(precision, amps, num_qubits, s,
						    kNoallocBlocks,
						    static_cast<cudaStream_t>(stream));
	return e == cudaSuccess ? DK_OK : DK_ERR_CUDA;
}
