// aem_dft.h -- launch interface of the time-series spectrum kernels (aem_dft.cu).
#pragma once
#include <cuda_runtime.h>

namespace aem {

constexpr long long DFT_RUN = 256;              // samples per chunk at least
constexpr int DFT_MAX_CHUNKS = 64;              // chunk sums per frequency at most
constexpr long long DFT_SCRATCH_COMPLEX = 65536;  // chunk sums (complex) the scratch must hold at most

// number of chunks the transform of n samples at nf frequencies uses
int dft_chunks(long long n, int nf);

// both passes on stream s; `scratch` holds 2 * chunks * nf doubles
cudaError_t dft_launch(const float* x, long long n, double dt, const double* freqs, int nf, double* out,
                       double* scratch, int chunks, cudaStream_t s);

// batched spectra of ns series (row stride ld, FP64 samples); `scratch`
// holds 2 * chunks * ns * nf doubles, out 2 * ns * nf (series-major)
int dftb_chunks(long long n, int ns, int nf);
cudaError_t dftb_launch(const double* x, long long ld, int ns, long long n, double dt, const double* freqs, int nf,
                        double* out, double* scratch, int chunks, cudaStream_t s);

}  // namespace aem
