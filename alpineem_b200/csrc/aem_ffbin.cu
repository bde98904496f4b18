// aem_ffbin.cu -- deterministic retarded-time binning of the far-field
// surface currents (FP32 runs), main_fdtd/fdtd_solver.f90:7643-7925 (and the
// image-plane pass :7929-8235).
//
// The reference adds, at every step n, each face cell's current difference
// dM = M - M_old into two bins of every angle:
//   t = n + 1/2 + tf - 1 (U, from M) or n + tf - 1 (W, from J),
//   U(ii) += (1-w) fac dM,  U(ii+1) += w fac dM,  ii = int(t), w = t - ii,
// with tf(cell, angle) the retarded-time offset, which does not change
// during the run.  Written with the bin offset k = floor(tf - 1/2) - 1
// (U; floor(tf) - 2 for W, 0-based bins) and w = frac(tf - 1/2) (frac(tf)),
// both fixed per (cell, angle), bin n + k receives
//   (1 - w) dM(n) + w dM(n - 1)
// from the cell: the contribution of step n and the carried-over part of
// step n - 1.  Here w and k are taken from tf once, exactly; the reference
// rounds n + 1/2 + tf in FP32 at every step, which moves w by up to half an
// ulp of n + tf (about 2.4e-4 at 4000 steps).
//
// Work of one batch of up to 32 steps:
//   k_ff_currents (aem_aux.cu) writes each step's differences to slot
//       1..32 of a tile-major buffer; slot 0 holds the step before the batch;
//   k_ff_bin_tiles: one CTA per (32x32 face tile, group of angles).  Lane t
//       of every warp owns step n0 + t, so a warp's 32 lanes always add to
//       32 different bins.  Each warp owns the histograms of its angles
//       (plain shared-memory adds, no atomics, fixed order), and the CTA
//       writes every (tile, angle) window to a partial buffer;
//   k_ff_reduce: one CTA per angle sums the windows of all tiles, faces and
//       image passes in a fixed order (tiles sorted by window base) in FP64
//       and adds them to FP64 accumulators: two runs give the same bits;
//   k_ff_carry: slot `nt` (the batch's last step) becomes slot 0 and slot 1
//       is cleared; a final one-lane pass with slot 1 = 0 adds the last
//       step's carried part.
#include "aem_dev.cuh"
#include "aem_kernels.h"

namespace aem {

namespace {

constexpr int BIN_WARPS = 8;
constexpr int STAGE_STRIDE = 4 * 33 + 1;  // floats per staged cell: 4 components x 33 slots, +1 (odd: no bank conflicts)
constexpr int STAGE_FLOATS = FF_TILE * STAGE_STRIDE;

// retarded-time offset of face cell (u, v), the same expression in every
// kernel that uses it
__device__ __forceinline__ float ff_tf(const float* k, float uf, float vf) { return fmaf(k[1], uf, fmaf(k[2], vf, k[0])); }

// bin offsets and weights of one (cell, angle): U from tf - 1/2 (exact in
// FP32 for the tf > 1 of every Huygens cell), W from tf
struct BinW {
    int ku, kw;
    float wu, ww;
};
__device__ __forceinline__ BinW ff_binw(float tf) {
    BinW r;
    const float xu = tf - 0.5f;
    const float fu = floorf(xu), fw = floorf(tf);
    r.wu = xu - fu;
    r.ww = tf - fw;
    r.ku = (int)fu - 1;
    r.kw = (int)fw - 2;
    return r;
}

// h + (w dd + d) on both lanes of a pair, rounded as fmaf then an add:
// packed FP32, one fma and one add for two histogram components
__device__ __forceinline__ float2 ff_acc2(float2 h, float w, float dd0, float dd1, float d0, float d1) {
    float2 r;
    asm("{\n .reg .b64 wa, xa, ya, pa, t;\n mov.b64 wa, {%2, %2};\n mov.b64 xa, {%3, %4};\n mov.b64 ya, {%5, %6};\n"
        " mov.b64 pa, {%7, %8};\n fma.rn.ftz.f32x2 t, wa, xa, ya;\n add.rn.ftz.f32x2 t, pa, t;\n mov.b64 {%0, %1}, t;\n}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(w), "f"(dd0), "f"(dd1), "f"(d0), "f"(d1), "f"(h.x), "f"(h.y));
    return r;
}

__device__ __forceinline__ void face_of_tile(const FarFieldDev& F, long long tile, int& f, int& u0, int& v0, int& nb,
                                             int& nc) {
    f = 0;
    while (f < 5 && tile >= F.tile0[f + 1]) f++;
    const int a = f >> 1;
    const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
    nb = F.hi[b] - F.lo[b] + 1;
    nc = F.hi[c] - F.lo[c] + 1;
    const long long tl = tile - F.tile0[f];
    u0 = (int)(tl % F.tiles_u[a]) * FF_TILE;
    v0 = (int)(tl / F.tiles_u[a]) * FF_TILE;
}

// setup: per (tile, angle) the lowest bin offset any of its cells reaches
// (the window base) and the span of offsets; one CTA per tile
__global__ void k_ff_base(const __grid_constant__ FarFieldDev F, int* kb, int* span) {
    const long long tile = blockIdx.x;
    int f, u0, v0, nb, nc;
    face_of_tile(F, tile, f, u0, v0, nb, nc);
    const int a = f >> 1, s = f & 1;
    const int nu = min(FF_TILE, nb - u0), nv = min(FF_TILE, nc - v0);
    int worst = 0;
    for (int j = threadIdx.x; j < F.nvc; j += blockDim.x) {
        const float* k = F.kf + (((long long)F.vlist[j] * 3 + a) * 2 + s) * 3;
        int lo = INT_MAX, hi = INT_MIN;
        for (int v = 0; v < nv; v++)
            for (int u = 0; u < nu; u++) {
                const BinW w = ff_binw(ff_tf(k, (float)(u0 + u), (float)(v0 + v)));
                lo = min(lo, min(w.ku, w.kw));
                hi = max(hi, max(w.ku, w.kw));
            }
        kb[tile * F.nvc + j] = lo;
        worst = max(worst, hi - lo);
    }
    if (worst) atomicMax(span, worst);
}

// One CTA per (face tile, group of F.group angles); see the file comment.
// AW angles per warp (F.group = BIN_WARPS * AW); TAIL: the run's last batch.
template <int AW, bool TAIL>
__global__ void __launch_bounds__(BIN_WARPS * 32, 2) k_ff_bin_tiles(const __grid_constant__ FarFieldDev F, int nlanes) {
    extern __shared__ __align__(16) float smem[];
    float* stage = smem;                                              // [2][32 cells][STAGE_STRIDE]
    float2* hist = reinterpret_cast<float2*>(smem + 2 * STAGE_FLOATS);  // [group][U, W][hs]
    const int HS = F.hs;
    const long long tile = blockIdx.y;
    int f, u0, v0, nb, nc;
    face_of_tile(F, tile, f, u0, v0, nb, nc);
    const int a = f >> 1, s = f & 1;
    const int nu = min(FF_TILE, nb - u0), nv = min(FF_TILE, nc - v0);
    const int j0 = blockIdx.x * F.group;
    const int ng = min(F.group, F.nvc - j0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int e = tid; e < ng * 2 * HS; e += blockDim.x) hist[e] = make_float2(0.0f, 0.0f);
    // this warp's angles: jl = warp + BIN_WARPS q
    float K0[AW], Ku[AW], Kv[AW];
    int base[AW];
#pragma unroll
    for (int q = 0; q < AW; q++) {
        const int jl = warp + BIN_WARPS * q;
        K0[q] = Ku[q] = Kv[q] = 0.0f;
        base[q] = 0;
        if (jl < ng) {
            const float* k = F.kf + (((long long)F.vlist[j0 + jl] * 3 + a) * 2 + s) * 3;
            K0[q] = k[0]; Ku[q] = k[1]; Kv[q] = k[2];
            base[q] = F.kb[tile * F.nvc + j0 + jl];
        }
    }

    // staging of one tile row: slots 0..nlanes of the 4 components of its
    // 32 cells, transposed to [cell][component][slot]
    const float* src = F.dtile + tile * FF_SLOTS * 4 * 1024;
    const int nrow4 = (nlanes + 1) * 4 * 8;  // float4 loads per row
    auto load_row = [&](int v, float4 (&r)[5]) {
#pragma unroll
        for (int q = 0; q < 5; q++) {
            const int e = tid + q * BIN_WARPS * 32;
            if (e < nrow4) r[q] = *reinterpret_cast<const float4*>(src + (long long)(e >> 3) * 1024 + v * 32 + (e & 7) * 4);
        }
    };
    auto store_row = [&](float* buf, const float4 (&r)[5]) {
#pragma unroll
        for (int q = 0; q < 5; q++) {
            const int e = tid + q * BIN_WARPS * 32;
            if (e < nrow4) {
                const int row = e >> 3, slot = row >> 2, m = row & 3, u = (e & 7) * 4;
                float* d = buf + u * STAGE_STRIDE + m * 33 + slot;
                d[0] = r[q].x;
                d[STAGE_STRIDE] = r[q].y;
                d[2 * STAGE_STRIDE] = r[q].z;
                d[3 * STAGE_STRIDE] = r[q].w;
            }
        }
    };
    float4 pre[5];
    load_row(0, pre);
    store_row(stage, pre);
    int bad = 0;
    const bool live = lane < nlanes;
    for (int v = 0; v < nv; v++) {
        float* cur = stage + (v & 1) * STAGE_FLOATS;
        if (v + 1 < nv) load_row(v + 1, pre);
        __syncthreads();  // row v staged; the other buffer's readers are done
        const float vf = (float)(v0 + v);
        float trow[AW];
#pragma unroll
        for (int q = 0; q < AW; q++) trow[q] = fmaf(Kv[q], vf, K0[q]);
        for (int u = 0; u < nu; u++) {
            const float* c = cur + u * STAGE_STRIDE;
            // lane t: d(n0 + t) (slot t + 1) and d(n0 + t - 1) (slot t)
            float d[4], dd[4];
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const float x1 = live ? c[m * 33 + lane + 1] : 0.0f;
                const float x0 = live ? c[m * 33 + lane] : 0.0f;
                d[m] = x1;
                dd[m] = x0 - x1;
            }
            const float uf = (float)(u0 + u);
            // every angle's bins first, then all histogram loads, adds and
            // stores: the angles' windows never overlap, so the loads of one
            // angle need not wait for the stores of another
            int iu[AW], iw[AW];
            float wu[AW], ww[AW];
            bool on[AW];
#pragma unroll
            for (int q = 0; q < AW; q++) {
                const BinW w = ff_binw(fmaf(Ku[q], uf, trow[q]));
                iu[q] = w.ku - base[q];
                iw[q] = w.kw - base[q];
                wu[q] = w.wu;
                ww[q] = w.ww;
                on[q] = warp + BIN_WARPS * q < ng;  // warp-uniform
                if (on[q] && ((unsigned)iu[q] > (unsigned)(HS - 33) || (unsigned)iw[q] > (unsigned)(HS - 33))) {
                    bad++;  // never: kb and hs come from the same expressions
                    on[q] = false;
                }
            }
            float2 pu[AW], pw[AW];
#pragma unroll
            for (int q = 0; q < AW; q++) {
                if (!on[q]) continue;
                const float2* h = hist + (warp + BIN_WARPS * q) * 2 * HS;
                pu[q] = h[iu[q] + lane];
                pw[q] = h[HS + iw[q] + lane];
            }
#pragma unroll
            for (int q = 0; q < AW; q++) {
                if (!on[q]) continue;
                pu[q] = ff_acc2(pu[q], wu[q], dd[0], dd[1], d[0], d[1]);
                pw[q] = ff_acc2(pw[q], ww[q], dd[2], dd[3], d[2], d[3]);
            }
#pragma unroll
            for (int q = 0; q < AW; q++) {
                if (!on[q]) continue;
                float2* h = hist + (warp + BIN_WARPS * q) * 2 * HS;
                h[iu[q] + lane] = pu[q];
                h[HS + iw[q] + lane] = pw[q];
            }
        }
        // the run's last batch: the carried part of the final step, w d(N),
        // of every cell of the row goes into the bin after that step's own
        // (what a batch of one step with zero differences would add there).
        // Lane u takes cell u; the cells of a row reach each bin in one
        // contiguous run (the offset is monotonic along the row), so a
        // masked shuffle sum gathers each run onto its first lane, which
        // alone adds it to the histogram.
        if (TAIL) {
            const bool cell = lane < nu;
            const float* c = cur + lane * STAGE_STRIDE;
            float dn[4];
#pragma unroll
            for (int m = 0; m < 4; m++) dn[m] = cell ? c[m * 33 + nlanes] : 0.0f;
            const float uf = (float)(u0 + lane);
#pragma unroll
            for (int q = 0; q < AW; q++) {
                if (warp + BIN_WARPS * q >= ng) continue;  // warp-uniform
                const BinW w = ff_binw(fmaf(Ku[q], uf, trow[q]));
                int key[2] = {cell ? w.ku - base[q] + nlanes : -1 - lane, cell ? w.kw - base[q] + nlanes : -1 - lane};
                float2 val[2] = {make_float2(fmaf(w.wu, dn[0], 0.0f), fmaf(w.wu, dn[1], 0.0f)),
                                 make_float2(fmaf(w.ww, dn[2], 0.0f), fmaf(w.ww, dn[3], 0.0f))};
#pragma unroll
                for (int h2 = 0; h2 < 2; h2++) {
#pragma unroll
                    for (int off = 1; off < 32; off <<= 1) {
                        const int ko = __shfl_down_sync(0xffffffffu, key[h2], off);
                        const float vx = __shfl_down_sync(0xffffffffu, val[h2].x, off);
                        const float vy = __shfl_down_sync(0xffffffffu, val[h2].y, off);
                        if (lane + off < 32 && ko == key[h2]) {
                            val[h2].x += vx;
                            val[h2].y += vy;
                        }
                    }
                    const int kp = __shfl_up_sync(0xffffffffu, key[h2], 1);
                    const bool head = cell && (lane == 0 || kp != key[h2]);
                    if (head) {
                        if ((unsigned)key[h2] > (unsigned)(HS - 1)) {
                            bad++;  // never: hs holds the span, the 32 lanes and this bin
                        } else {
                            float2* hh = hist + (warp + BIN_WARPS * q) * 2 * HS + h2 * HS;
                            float2 t = hh[key[h2]];
                            t.x += val[h2].x;
                            t.y += val[h2].y;
                            hh[key[h2]] = t;
                        }
                    }
                }
            }
        }
        if (v + 1 < nv) store_row(stage + ((v + 1) & 1) * STAGE_FLOATS, pre);
    }
    if (bad && lane == 0) atomicAdd(F.err, bad);
    __syncthreads();
    // windows -> partial buffer [tile][j][m][hs]; m = 0 U1, 1 U2, 2 W1, 3 W2
    const float* hf = reinterpret_cast<const float*>(hist);
    for (int e = tid; e < ng * 4 * HS; e += blockDim.x) {
        const int jl = e / (4 * HS), r = e % (4 * HS), m = r / HS, k = r % HS;
        // hist layout per angle: [U, W][hs] pairs (x: comp 1, y: comp 2)
        const float val = hf[((jl * 2 + (m >> 1)) * HS + k) * 2 + (m & 1)];
        F.part[((tile * F.nvc + j0 + jl) * 4 + m) * HS + k] = val;
    }
}

// Ordered reduction of the windows of one batch into the FP64 accumulators.
// One CTA per binned angle; element (component X, bin offset r) sums, in
// this fixed order, the image passes, the faces whose tangential axes carry
// X, and the tiles of each face in (kb, tile) order.
__global__ void k_ff_reduce(const __grid_constant__ AemParams P, const __grid_constant__ FarFieldDev F, int n0, int nt) {
    if (P.dstep) n0 = *P.dstep - nt + 1;  // graph replay: the batch ends at the current step
    const int ci = blockIdx.x;
    const int* cl = F.clist + 4 * ci;
    const int ang = cl[0];
    const int lo = F.crange[2 * ci], hi = F.crange[2 * ci + 1];
    const int R = hi - lo, HS = F.hs;
    double* UW = reinterpret_cast<double*>(F.UW);
    for (long long e = threadIdx.x; e < 6LL * R; e += blockDim.x) {
        const int X = (int)(e / R), r = lo + (int)(e % R);
        const int x = X % 3;  // Cartesian axis of the component; X < 3: W, else U
        double acc = 0.0;
        for (int pass = 0; pass <= F.mirror; pass++) {
            const int j = cl[1 + pass];
            if (j < 0) continue;
            for (int fa = 0; fa < 3; fa++) {
                if (fa == x || !F.has[fa] || !F.face_n[fa]) continue;
                const int b = fa == 0 ? 1 : 0;
                const int first = x == b ? 0 : 1;  // U1/W1 carry axis b, U2/W2 axis c
                const int m = (X >= 3 ? 0 : 2) + first;
                float sg = 1.0f;
                if (pass) sg = m == 0 || m == 1 ? F.M_mir[x] : F.J_mir[x];
                const double fac = (double)(F.fac[fa] * sg);
                for (int side = 0; side < 2; side++) {
                    const int f = 2 * fa + side;
                    const int nt_f = (int)(F.tile0[f + 1] - F.tile0[f]);
                    const int* lst = F.srt + ((long long)j * 6 + f) * F.maxt;
                    const int* kbl = F.srtkb + ((long long)j * 6 + f) * F.maxt;
                    // first tile whose window reaches r: kb > r - HS
                    int l = 0, h = nt_f;
                    while (l < h) {
                        const int mid = (l + h) >> 1;
                        if (kbl[mid] > r - HS) h = mid;
                        else l = mid + 1;
                    }
                    double sub = 0.0;
                    for (int q = l; q < nt_f && kbl[q] <= r; q++)
                        sub += (double)F.part[(((long long)lst[q] * F.nvc + j) * 4 + m) * HS + (r - kbl[q])];
                    acc += sub * fac;
                }
            }
        }
        const long long gb = (long long)n0 + r;
        if (gb < 0 || gb >= F.len) {
            if (acc != 0.0) atomicAdd(F.err, 1);
            continue;
        }
        UW[((long long)X * F.nang + ang) * F.len + gb] += acc;
    }
}

// slot `carry` -> slot 0, slot 1 cleared, over every tile cell
__global__ void k_ff_carry(const __grid_constant__ FarFieldDev F, int carry) {
    const long long n = (long long)F.ntiles * 4 * 1024;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long t = e / (4 * 1024), r = e % (4 * 1024);
        float* d = F.dtile + t * FF_SLOTS * 4 * 1024 + r;
        d[0] = d[(long long)carry * 4 * 1024];
        d[4 * 1024] = 0.0f;
    }
}

template <int AW>
void bin_launch(const FarFieldDev& F, int nlanes, bool tail, cudaStream_t s) {
    dim3 grid((unsigned)F.ngrp, (unsigned)F.ntiles);
    if (tail) k_ff_bin_tiles<AW, true><<<grid, BIN_WARPS * 32, ff_tiles_smem(F), s>>>(F, nlanes);
    else k_ff_bin_tiles<AW, false><<<grid, BIN_WARPS * 32, ff_tiles_smem(F), s>>>(F, nlanes);
}

}  // namespace

size_t ff_tiles_smem(const FarFieldDev& F) {
    return (size_t)2 * STAGE_FLOATS * sizeof(float) + (size_t)F.group * 2 * F.hs * sizeof(float2);
}

void ff_tiles_prepare() {
    const int lim = 200 * 1024;
    cudaFuncSetAttribute(k_ff_bin_tiles<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_ff_bin_tiles<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_ff_bin_tiles<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_ff_bin_tiles<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_ff_bin_tiles<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(k_ff_bin_tiles<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

int launch_ff_base(const FarFieldDev& F, int* kb, int* span, cudaStream_t s) {
    if (!F.ntiles || !F.nvc) return 0;
    k_ff_base<<<(unsigned)F.ntiles, 128, 0, s>>>(F, kb, span);
    return 1;
}

int launch_ff_bin_tiles(const AemParams& P, const FarFieldDev& F, int n0, int nlanes, int carry, cudaStream_t s,
                        bool tail) {
    if (!F.nvc || !F.ntiles || nlanes <= 0) return 0;
    const int aw = F.group / BIN_WARPS;
    if (aw >= 4) bin_launch<4>(F, nlanes, tail, s);
    else if (aw == 2) bin_launch<2>(F, nlanes, tail, s);
    else bin_launch<1>(F, nlanes, tail, s);
    k_ff_reduce<<<(unsigned)F.nangc, 256, 0, s>>>(P, F, n0, nlanes);
    int n = 2;
    if (carry > 0) {
        const long long tot = (long long)F.ntiles * 4 * 1024;
        const int blocks = (int)std::min<long long>((tot + 255) / 256, 148 * 16);
        k_ff_carry<<<blocks, 256, 0, s>>>(F, carry);
        n++;
    }
    return n;
}

}  // namespace aem
