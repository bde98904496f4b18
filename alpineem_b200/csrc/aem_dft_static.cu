// aem_dft_static.cu -- aem_dft_static: the spectrum of aem_dft without any
// device allocation, for callers that cannot allocate device memory.
//
// Some hosts own every byte of device memory themselves: an application
// that reserves the GPU's memory up front in its own arena, a plugin
// interface whose callbacks must not allocate, or a real-time loop where an
// allocation could block or fail at the wrong moment.  aem_dft takes its
// chunk-sum buffer from the stream-ordered pool on every call; this entry
// point instead uses one fixed array in the library's device image,
// `g_dft_scratch`, sized for DFT_SCRATCH_COMPLEX complex chunk sums (1 MiB).
// Every GPU that loads the library holds that megabyte until the process
// exits.  The caller passes the input series, the frequencies and the output
// buffer, all device memory it owns.
//
// Host code cannot pass `g_dft_scratch` to a kernel by name: on the host
// the name denotes a stand-in object, not a device address.  The device
// address is looked up with cudaGetSymbolAddress once per device, on the
// first call made while that device is current, and cached for the life of
// the process.  The cache assumes the device's primary context lives that
// long: after cudaDeviceReset (or any teardown of the primary context) the
// array may sit at another address, so a process that resets a device must
// not call aem_dft_static on it again.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/alpineem_b200.h"
#include "aem_dft.h"

namespace aem {
void set_global_error(const std::string& msg);  // aem_api.cpp
}

namespace {

__device__ __align__(256) double g_dft_scratch[2 * aem::DFT_SCRATCH_COMPLEX];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

int fail(int code, const std::string& msg) {
    aem::set_global_error(msg);
    return code;
}

}  // namespace

extern "C" int aem_dft_static(const float* x, long long n, double dt, const double* freqs, int nf, double* out,
                              void* stream) {
    if (!x || !freqs || !out || n < 1 || nf < 1 || !(dt > 0.0)) return fail(AEM_ERR_ARG, "bad argument");
    if ((long long)nf > aem::DFT_SCRATCH_COMPLEX)
        return fail(AEM_ERR_ARG, "aem_dft_static: " + std::to_string(nf) + " frequencies exceed the static scratch (at most " +
                                     std::to_string(aem::DFT_SCRATCH_COMPLEX) + ")");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return fail(AEM_ERR_CUDA, "CUDA error: no usable CUDA device");
    }
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_dft_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                return fail(AEM_ERR_CUDA, std::string("CUDA error: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            }
            g_scratch_addr[dev] = static_cast<double*>(p);
        }
        scratch = g_scratch_addr[dev];
    }
    // the same chunking as aem_dft; it never needs more than the array holds.
    // The first pass writes every chunk sum the second pass reads, so the
    // previous call's contents need no clearing.
    const int chunks = aem::dft_chunks(n, nf);
    if ((long long)chunks * nf > aem::DFT_SCRATCH_COMPLEX) return fail(AEM_ERR_ARG, "aem_dft_static: scratch too small");
    e = aem::dft_launch(x, n, dt, freqs, nf, out, scratch, chunks, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(AEM_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    }
    return AEM_OK;
}
