// aem_dft.cu -- spectrum of a time series at arbitrary frequencies on the GPU:
//   X(f) = sum_{m=0}^{n-1} x[m] exp(-i 2 pi f m dt).
//
// This is what utility_scripts/post_processor.py gets from numpy's FFT of
// the zero-padded series (post_processor.py:160-215): the padded FFT bin k
// is X(k / (N dt)) with N = (padding+1) n.  Evaluating X directly at the
// wanted frequencies (e.g. the 512 S11 frequencies of a run) needs no
// padding.  Two passes, both deterministic:
//   1. k_dft_partial: the samples are cut into `chunks` equal runs; thread f
//      of CTA column c sums run c for frequency f in FP64 (phase reduced to
//      [0, 2) half-turns before sincospi, so long runs keep full accuracy);
//   2. k_dft_reduce: one thread per frequency adds the chunk sums in order.
// The chunk sums live in a scratch buffer of chunks * nf complex doubles.
#include <cuda_runtime.h>

#include "aem_dft.h"

namespace aem {

int dft_chunks(long long n, int nf) {
    long long c = (n + DFT_RUN - 1) / DFT_RUN;
    if (c > DFT_MAX_CHUNKS) c = DFT_MAX_CHUNKS;
    const long long cap = nf > 0 ? DFT_SCRATCH_COMPLEX / nf : 1;
    if (c > cap) c = cap;
    return c < 1 ? 1 : (int)c;
}

__global__ void k_dft_partial(const float* __restrict__ x, long long n, double dt, const double* __restrict__ freqs,
                              int nf, int chunks, double* __restrict__ part) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int chunk = blockIdx.y;
    if (f >= nf) return;
    const long long len = (n + chunks - 1) / chunks;
    const long long m0 = (long long)chunk * len;
    const long long m1 = m0 + len < n ? m0 + len : n;
    const double a = 2.0 * freqs[f] * dt;  // phase advance per sample, in half-turns
    double re = 0.0, im = 0.0;
    for (long long m = m0; m < m1; m++) {
        double ph = a * (double)m;
        ph -= 2.0 * floor(0.5 * ph);
        double s, c;
        sincospi(ph, &s, &c);
        const double v = (double)x[m];
        re += v * c;
        im -= v * s;
    }
    part[2 * ((long long)chunk * nf + f)] = re;
    part[2 * ((long long)chunk * nf + f) + 1] = im;
}

__global__ void k_dft_reduce(const double* __restrict__ part, int nf, int chunks, double* __restrict__ out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    double re = 0.0, im = 0.0;
    for (int c = 0; c < chunks; c++) {
        re += part[2 * ((long long)c * nf + f)];
        im += part[2 * ((long long)c * nf + f) + 1];
    }
    out[2 * f] = re;
    out[2 * f + 1] = im;
}

cudaError_t dft_launch(const float* x, long long n, double dt, const double* freqs, int nf, double* out,
                       double* scratch, int chunks, cudaStream_t s) {
    const int T = 128;
    dim3 g1((nf + T - 1) / T, chunks);
    k_dft_partial<<<g1, T, 0, s>>>(x, n, dt, freqs, nf, chunks, scratch);
    k_dft_reduce<<<(nf + T - 1) / T, T, 0, s>>>(scratch, nf, chunks, out);
    return cudaGetLastError();
}

}  // namespace aem
