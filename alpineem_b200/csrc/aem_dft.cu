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

// ---------------------------------------------------------------------------
// Batched spectra of many series sampled alike (every far-field angle and
// polarisation, the ports, the incident wave of a run):
//   X[s][f] = sum_{m=0}^{n-1} x[s*ld + m] exp(-i 2 pi f m dt).
// Thread f of a CTA holds DFTB_SERIES accumulators; the samples of those
// series arrive in shared-memory tiles read by every thread, so the twiddle
// of (f, m) is computed once for DFTB_SERIES series.  The sample range may
// be cut into chunks (grid y) summed afterwards in chunk order, so results
// do not depend on scheduling.
namespace aem {
namespace {
constexpr int DFTB_SERIES = 8, DFTB_TILE = 256, DFTB_T = 128;

__global__ void __launch_bounds__(DFTB_T) k_dftb_partial(const double* __restrict__ x, long long ld, int ns, long long n,
                                                         double dt, const double* __restrict__ freqs, int nf, int chunks,
                                                         double* __restrict__ part) {
    __shared__ double tile[DFTB_SERIES][DFTB_TILE];
    const int f = blockIdx.x * DFTB_T + threadIdx.x;
    const int s0 = blockIdx.z * DFTB_SERIES;
    const int chunk = blockIdx.y;
    const long long len = (n + chunks - 1) / chunks;
    const long long m0 = (long long)chunk * len, m1 = m0 + len < n ? m0 + len : n;
    const double a = f < nf ? 2.0 * freqs[f] * dt : 0.0;  // half-turns per sample
    double re[DFTB_SERIES], im[DFTB_SERIES];
    for (int q = 0; q < DFTB_SERIES; q++) re[q] = im[q] = 0.0;
    for (long long t0 = m0; t0 < m1; t0 += DFTB_TILE) {
        const int tl = (int)(m1 - t0 < DFTB_TILE ? m1 - t0 : DFTB_TILE);
        __syncthreads();
        for (int e = threadIdx.x; e < DFTB_SERIES * DFTB_TILE; e += DFTB_T) {
            const int q = e / DFTB_TILE, m = e % DFTB_TILE;
            tile[q][m] = (s0 + q < ns && m < tl) ? x[(long long)(s0 + q) * ld + t0 + m] : 0.0;
        }
        __syncthreads();
        if (f < nf)
            for (int m = 0; m < tl; m++) {
                double ph = a * (double)(t0 + m);
                ph -= 2.0 * floor(0.5 * ph);
                double sn, cs;
                sincospi(ph, &sn, &cs);
#pragma unroll
                for (int q = 0; q < DFTB_SERIES; q++) {
                    const double v = tile[q][m];
                    re[q] += v * cs;
                    im[q] -= v * sn;
                }
            }
    }
    if (f >= nf) return;
    for (int q = 0; q < DFTB_SERIES; q++) {
        if (s0 + q >= ns) break;
        const long long o = 2 * (((long long)chunk * ns + s0 + q) * nf + f);
        part[o] = re[q];
        part[o + 1] = im[q];
    }
}

__global__ void k_dftb_reduce(const double* __restrict__ part, int ns, int nf, int chunks, double* __restrict__ out) {
    const long long tot = (long long)ns * nf;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        double re = 0.0, im = 0.0;
        for (int c = 0; c < chunks; c++) {
            re += part[2 * ((long long)c * tot + e)];
            im += part[2 * ((long long)c * tot + e) + 1];
        }
        out[2 * e] = re;
        out[2 * e + 1] = im;
    }
}
}  // namespace

int dftb_chunks(long long n, int ns, int nf) {
    // enough CTAs for every SM several times over, each chunk at least
    // DFTB_TILE samples
    const long long ctas = (long long)((nf + DFTB_T - 1) / DFTB_T) * ((ns + DFTB_SERIES - 1) / DFTB_SERIES);
    long long c = (148LL * 8 + ctas - 1) / ctas;
    const long long cmax = (n + DFTB_TILE - 1) / DFTB_TILE;
    if (c > cmax) c = cmax;
    if (c > 64) c = 64;
    return c < 1 ? 1 : (int)c;
}

cudaError_t dftb_launch(const double* x, long long ld, int ns, long long n, double dt, const double* freqs, int nf,
                        double* out, double* scratch, int chunks, cudaStream_t s) {
    dim3 g((nf + DFTB_T - 1) / DFTB_T, chunks, (ns + DFTB_SERIES - 1) / DFTB_SERIES);
    if (g.z > 65535) return cudaErrorInvalidValue;
    k_dftb_partial<<<g, DFTB_T, 0, s>>>(x, ld, ns, n, dt, freqs, nf, chunks, scratch);
    const long long tot = (long long)ns * nf;
    const int blocks = (int)((tot + 255) / 256 < 148 * 16 ? (tot + 255) / 256 : 148 * 16);
    k_dftb_reduce<<<blocks, 256, 0, s>>>(scratch, ns, nf, chunks, out);
    return cudaGetLastError();
}

}  // namespace aem
