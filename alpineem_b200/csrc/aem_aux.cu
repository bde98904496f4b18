// aem_aux.cu -- the small per-step kernels around the two field updates:
// lumped ports, far-field Huygens currents and retarded-time binning,
// unit-cell plane sums, phase-centre samples and 2-D video slices.
#include "aem_dev.cuh"
#include "aem_kernels.h"

namespace aem {

template <typename T>
__device__ inline T& at(void* base, long long i) {
    return reinterpret_cast<T*>(base)[i];
}

// storage position of a reference index (wraps on periodic axes)
__device__ inline int pidx(const AemParams& P, int a, int idx) {
    if (P.per[a]) {
        const int n = a == 0 ? P.SX : a == 1 ? P.SY : P.SZ;
        int p = (idx - 1) % n;
        return p < 0 ? p + n : p;
    }
    return idx - 1;
}
__device__ inline long long cidx(const AemParams& P, int i, int j, int k) {
    return lin(P, pidx(P, 0, i), pidx(P, 1, j), pidx(P, 2, k));
}
// field value at reference indices; on a periodic axis an index past the
// stored period carries the Bloch phase (kmax)
template <typename T>
__device__ inline T fget(const AemParams& P, const void* F, int i, int j, int k) {
    T v = reinterpret_cast<const T*>(F)[cidx(P, i, j, k)];
    const int idx[3] = {i, j, k};
    const int S[3] = {P.SX, P.SY, P.SZ};
    for (int a = 0; a < 3; a++) {
        if (!P.per[a]) continue;
        if (idx[a] > S[a]) v = bloch<T>(v, P, a, -1);
        if (idx[a] < 1) v = bloch<T>(v, P, a, +1);
    }
    return v;
}
__device__ inline float feed(const PortDev& p, int c, int a, int b) {
    return p.feed[((long long)(b - 1) * (p.n1 + 1) + (a - 1)) * 4 + (c - 1)];
}

// ports on the H half-step, ref :4800-5118
template <typename T>
__global__ void k_ports_h(const __grid_constant__ AemParams P, const __grid_constant__ PortSet S, int counter) {
    counter = step_of(P, counter);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int n = 0; n < S.n; n++) {
            const PortDev& p = S.p[n];
            T cur = zero<T>();
            const int p1 = p.loc[0], p2 = p.loc[1], p3 = p.loc[2];
            if (!p.gridded) {  // loop current around the port, ref :4820-4857
                const int d1 = p.size[0] + p1 - 1, d2 = p.size[1] + p2 - 1, d3 = p.size[2] + p3 - 1;
                if (p.dir == 0) {
                    for (int a = p1; a <= d1; a++) {
                        for (int b = p2; b <= d2; b++) cur = cur + p.dl[1] * (fget<T>(P, P.H[1], a, b, p3 - 1) - fget<T>(P, P.H[1], a, b, d3));
                        for (int c = p3; c <= d3; c++) cur = cur + p.dl[2] * (fget<T>(P, P.H[2], a, p2, c) - fget<T>(P, P.H[2], a, d2 - 1, c));
                    }
                    cur = cur * (p.sizef[1] * p.sizef[2]) / p.sizef[0];
                } else if (p.dir == 1) {
                    for (int b = p2; b <= d2; b++) {
                        for (int a = p1; a <= d1; a++) cur = cur + p.dl[0] * (fget<T>(P, P.H[0], a, b, p3) - fget<T>(P, P.H[0], a, b, d3 - 1));
                        for (int c = p3; c <= d3; c++) cur = cur + p.dl[2] * (fget<T>(P, P.H[2], p1 - 1, b, c) - fget<T>(P, P.H[2], d1, b, c));
                    }
                    cur = cur * (p.sizef[0] * p.sizef[2]) / p.sizef[1];
                } else {
                    for (int c = p3; c <= d3; c++) {
                        for (int a = p1; a <= d1; a++) cur = cur + p.dl[0] * (fget<T>(P, P.H[0], a, p2 - 1, c) - fget<T>(P, P.H[0], a, d2, c));
                        for (int b = p2; b <= d2; b++) cur = cur + p.dl[1] * (fget<T>(P, P.H[1], p1, b, c) - fget<T>(P, P.H[1], d1 - 1, b, c));
                    }
                    cur = cur * (p.sizef[0] * p.sizef[1]) / p.sizef[2];
                }
            } else {  // TEM mode projection, ref :4862-4954
                for (int a = 1; a <= p.n1 + 1; a++)
                    for (int b = 1; b <= p.n2 + 1; b++) {
                        const float g3 = feed(p, 3, a, b), g4 = feed(p, 4, a, b);
                        T h1, h2;
                        switch (p.side) {
                        case 0: h1 = fget<T>(P, P.H[1], p1 - 1, a + p2 - 1, b + p3 - 1); h2 = fget<T>(P, P.H[2], p1 - 1, a + p2 - 1, b + p3 - 1); break;
                        case 1: h1 = fget<T>(P, P.H[1], p1, a + p2 - 1, b + p3 - 1); h2 = fget<T>(P, P.H[2], p1, a + p2 - 1, b + p3 - 1); break;
                        case 2: h1 = fget<T>(P, P.H[0], p1 + a - 1, p2 - 1, b + p3 - 1); h2 = fget<T>(P, P.H[2], p1 + a - 1, p2 - 1, b + p3 - 1); break;
                        case 3: h1 = fget<T>(P, P.H[0], p1 + a - 1, p2, b + p3 - 1); h2 = fget<T>(P, P.H[2], p1 + a - 1, p2, b + p3 - 1); break;
                        case 4: h1 = fget<T>(P, P.H[0], p1 + a - 1, p2 + b - 1, p3 - 1); h2 = fget<T>(P, P.H[1], p1 + a - 1, p2 + b - 1, p3 - 1); break;
                        default: h1 = fget<T>(P, P.H[0], p1 + a - 1, p2 + b - 1, p3); h2 = fget<T>(P, P.H[1], p1 + a - 1, p2 + b - 1, p3); break;
                        }
                        cur = cur + h1 * g3 + h2 * g4;
                    }
                if (p.side == 0 || p.side == 3 || p.side == 4) cur = cur * -1.0f;
                cur = cur / p.feed_norm;
            }
            at<T>(p.I, 0) = cur;
        }
    }
    __syncthreads();
    // 1-D line currents, ref :4961-4983
    for (int n = 0; n < S.n; n++) {
        const PortDev& p = S.p[n];
        for (int j = 2 + tid; j <= S.P - 1; j += blockDim.x)
            at<T>(p.I, j - 1) = at<T>(p.I, j - 1) - p.cI * (at<T>(p.V, j) - at<T>(p.V, j - 1));
    }
    __syncthreads();
    if (tid == 0) {
        for (int n = 0; n < S.n; n++) {  // current source, ref :4987-5011
            const PortDev& p = S.p[n];
            if (p.excite) at<T>(p.I, 1) = at<T>(p.I, 1) - p.cI * reinterpret_cast<const T*>(S.srcI)[counter - 1];
        }
        for (int n = 0; n < S.n; n++) {  // zero H behind gridded ports, ref :5018-5116
            const PortDev& p = S.p[n];
            if (!p.gridded) continue;
            const int p1 = p.loc[0], p2 = p.loc[1], p3 = p.loc[2];
            for (int a = 1; a <= p.n1 + 1; a++)
                for (int b = 1; b <= p.n2 + 1; b++) {
                    const bool z3 = feed(p, 3, a, b) != 0.0f, z4 = feed(p, 4, a, b) != 0.0f;
                    void *F1, *F2;
                    int i1, j1, k1;
                    switch (p.side) {
                    case 0: F1 = P.H[1]; F2 = P.H[2]; i1 = p1; j1 = a + p2 - 1; k1 = b + p3 - 1; break;
                    case 1: F1 = P.H[1]; F2 = P.H[2]; i1 = p1 - 1; j1 = a + p2 - 1; k1 = b + p3 - 1; break;
                    case 2: F1 = P.H[0]; F2 = P.H[2]; i1 = p1 + a - 1; j1 = p2; k1 = b + p3 - 1; break;
                    case 3: F1 = P.H[0]; F2 = P.H[2]; i1 = p1 + a - 1; j1 = p2 - 1; k1 = b + p3 - 1; break;
                    case 4: F1 = P.H[0]; F2 = P.H[1]; i1 = p1 + a - 1; j1 = p2 + b - 1; k1 = p3; break;
                    default: F1 = P.H[0]; F2 = P.H[1]; i1 = p1 + a - 1; j1 = p2 + b - 1; k1 = p3 - 1; break;
                    }
                    if (z3) at<T>(F1, cidx(P, i1, j1, k1)) = zero<T>();
                    if (z4) at<T>(F2, cidx(P, i1, j1, k1)) = zero<T>();
                }
        }
    }
}

// ports on the E half-step, ref :6123-6283, plus the voltage tap :8241
template <typename T>
__global__ void k_ports_e(const __grid_constant__ AemParams P, const __grid_constant__ PortSet S, int counter) {
    counter = step_of(P, counter);
    const int tid = threadIdx.x;
    for (int n = 0; n < S.n; n++) {  // 1-D line voltages, ref :6125-6142
        const PortDev& p = S.p[n];
        for (int j = 2 + tid; j <= S.P - 1; j += blockDim.x)
            at<T>(p.V, j - 1) = at<T>(p.V, j - 1) - p.cV * (at<T>(p.I, j - 1) - at<T>(p.I, j - 2));
    }
    __syncthreads();
    if (tid != 0) return;
    for (int n = 0; n < S.n; n++) {  // voltage source, ref :6148-6172
        const PortDev& p = S.p[n];
        if (p.excite) at<T>(p.V, 1) = at<T>(p.V, 1) + p.cS * reinterpret_cast<const T*>(S.srcV)[counter - 1];
    }
    for (int n = 0; n < S.n; n++) {  // E at the port, ref :6178-6281
        const PortDev& p = S.p[n];
        const T v2 = at<T>(p.V, 1);
        const int p1 = p.loc[0], p2 = p.loc[1], p3 = p.loc[2];
        if (!p.gridded) {
            const int d1 = p.size[0] + p1 - 1, d2 = p.size[1] + p2 - 1, d3 = p.size[2] + p3 - 1;
            const T e = 1.0f * v2 / (p.sizef[p.dir] * p.dl[p.dir]);
            for (int a = p1; a <= d1; a++)
                for (int b = p2; b <= d2; b++)
                    for (int c = p3; c <= d3; c++) at<T>(P.E[p.dir], cidx(P, a, b, c)) = e;
        } else {
            for (int a = 1; a <= p.n1 + 1; a++)
                for (int b = 1; b <= p.n2 + 1; b++) {
                    const float g1 = feed(p, 1, a, b), g2 = feed(p, 2, a, b);
                    if (p.side <= 1) {
                        if (g1 != 0.0f) at<T>(P.E[1], cidx(P, p1, a + p2 - 1, b + p3 - 1)) = v2 * g1;
                        if (g2 != 0.0f) at<T>(P.E[2], cidx(P, p1, a + p2 - 1, b + p3 - 1)) = v2 * g2;
                    } else if (p.side <= 3) {
                        if (g1 != 0.0f) at<T>(P.E[0], cidx(P, p1 + a - 1, p2, b + p3 - 1)) = v2 * g1;
                        if (g2 != 0.0f) at<T>(P.E[2], cidx(P, p1 + a - 1, p2, b + p3 - 1)) = v2 * g2;
                    } else {
                        if (g1 != 0.0f) at<T>(P.E[0], cidx(P, p1 + a - 1, p2 + b - 1, p3)) = v2 * g1;
                        if (g2 != 0.0f) at<T>(P.E[1], cidx(P, p1 + a - 1, p2 + b - 1, p3)) = v2 * g2;
                    }
                }
        }
        at<T>(p.vout, counter - 1) = v2;
    }
}

// ---------------------------------------------------------------------------
// Huygens-surface currents, ref :7512-7641 (standard) and :7202-7331 (kmax,
// Bloch phase removed).  Face (a,s): cells over the two other axes (b<c);
// 8 arrays per face: 4 current components then their previous values.
template <typename T>
__device__ inline T unphase(const AemParams& P, const FarFieldDev& F, T v, int i, int j, int k, int a);
template <>
__device__ inline float unphase<float>(const AemParams&, const FarFieldDev&, float v, int, int, int, int) { return v; }
template <>
__device__ inline cf unphase<cf>(const AemParams& P, const FarFieldDev& F, cf v, int i, int j, int k, int a) {
    float ph;
    if (a == 0) ph = F.kc3[2] * (float)(k - F.kc) * P.del[2] + F.kc3[1] * (float)(j - F.jc) * P.del[1];
    else if (a == 1) ph = F.kc3[2] * (float)(k - F.kc) * P.del[2] + F.kc3[0] * (float)(i - F.ic) * P.del[0];
    else ph = F.kc3[1] * (float)(j - F.jc) * P.del[1] + F.kc3[0] * (float)(i - F.ic) * P.del[0];
    float s, c;
    sincosf(ph, &s, &c);
    return cmul(v, cf{c, -s});
}

template <typename T>
__global__ void k_ff_currents(const __grid_constant__ AemParams P, const __grid_constant__ FarFieldDev F, int slot) {
    const long long tot = 2 * (F.face_n[0] + F.face_n[1] + F.face_n[2]);
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < tot; g += (long long)gridDim.x * blockDim.x) {
        long long r = g;
        int a = 0;
        while (r >= 2 * F.face_n[a]) { r -= 2 * F.face_n[a]; a++; }
        const int s = (int)(r / F.face_n[a]);
        const long long q = r % F.face_n[a];
        const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
        const int nb = F.hi[b] - F.lo[b] + 1;
        int idx[3];
        idx[a] = s ? F.hi[a] : F.lo[a];
        idx[b] = F.lo[b] + (int)(q % nb);
        idx[c] = F.lo[c] + (int)(q / nb);
        const int i = idx[0], j = idx[1], k = idx[2];
        const float w = s ? F.wall_hi[a] : F.wall_lo[a];
        const float sg = s ? -1.0f : 1.0f;  // the high face flips every component
        T v[4];
        const void *Ex = P.E[0], *Ey = P.E[1], *Ez = P.E[2], *Hx = P.H[0], *Hy = P.H[1], *Hz = P.H[2];
        if (a == 0) {
            v[0] = (-1.0f * sg) * ((fget<T>(P, Ez, i, j, k) + fget<T>(P, Ez, i, j + 1, k) + fget<T>(P, Ez, i + 1, j, k) + fget<T>(P, Ez, i + 1, j + 1, k)) / 4.0f) * w;
            v[1] = sg * ((fget<T>(P, Ey, i, j, k) + fget<T>(P, Ey, i + 1, j, k) + fget<T>(P, Ey, i, j, k + 1) + fget<T>(P, Ey, i + 1, j, k + 1)) / 4.0f) * w;
            v[2] = sg * ((fget<T>(P, Hz, i, j, k) + fget<T>(P, Hz, i, j, k + 1)) / 2.0f) * w;
            v[3] = (-1.0f * sg) * ((fget<T>(P, Hy, i, j, k) + fget<T>(P, Hy, i, j + 1, k)) / 2.0f) * w;
        } else if (a == 1) {
            v[0] = sg * ((fget<T>(P, Ez, i, j, k) + fget<T>(P, Ez, i + 1, j, k) + fget<T>(P, Ez, i, j + 1, k) + fget<T>(P, Ez, i + 1, j + 1, k)) / 4.0f) * w;
            v[1] = (-1.0f * sg) * ((fget<T>(P, Ex, i, j, k) + fget<T>(P, Ex, i, j + 1, k) + fget<T>(P, Ex, i, j, k + 1) + fget<T>(P, Ex, i, j + 1, k + 1)) / 4.0f) * w;
            v[2] = (-1.0f * sg) * ((fget<T>(P, Hz, i, j, k) + fget<T>(P, Hz, i, j, k + 1)) / 2.0f) * w;
            v[3] = sg * ((fget<T>(P, Hx, i, j, k) + fget<T>(P, Hx, i + 1, j, k)) / 2.0f) * w;
        } else {
            v[0] = (-1.0f * sg) * ((fget<T>(P, Ey, i, j, k) + fget<T>(P, Ey, i + 1, j, k) + fget<T>(P, Ey, i, j, k + 1) + fget<T>(P, Ey, i + 1, j, k + 1)) / 4.0f) * w;
            v[1] = sg * ((fget<T>(P, Ex, i, j, k) + fget<T>(P, Ex, i, j + 1, k) + fget<T>(P, Ex, i, j, k + 1) + fget<T>(P, Ex, i, j + 1, k + 1)) / 4.0f) * w;
            v[2] = sg * ((fget<T>(P, Hy, i, j, k) + fget<T>(P, Hy, i, j + 1, k)) / 2.0f) * w;
            v[3] = (-1.0f * sg) * ((fget<T>(P, Hx, i, j, k) + fget<T>(P, Hx, i + 1, j, k)) / 2.0f) * w;
        }
        T* cur = reinterpret_cast<T*>(F.cur[a][s]);
        const long long n = F.face_n[a];
        // tiled difference buffer of the batched binning: tile of (u, v),
        // slot `slot` (1-based step of the batch); a complex run keeps the
        // imaginary parts in a second plane after the real ones
        const int u = (int)(q % nb), vv = (int)(q / nb);
        const long long tile = F.tile0[2 * a + s] + (u >> 5) + (long long)(vv >> 5) * F.tiles_u[a];
        float* dt = F.dtile + (tile * FF_SLOTS + slot) * 4 * 1024 + ((vv & 31) << 5) + (u & 31);
        for (int m = 0; m < 4; m++) {
            if constexpr (sizeof(T) == sizeof(float)) {
                const float nv = v[m];
                dt[m * 1024] = nv - cur[m * n + q];  // M - M_o, ref :7667
                cur[m * n + q] = nv;
            } else {
                const T nv = unphase<T>(P, F, v[m], i, j, k, a);  // ref :7202-7331
                const T df = nv - cur[m * n + q];
                const long long plane = (long long)F.ntiles * FF_SLOTS * 4 * 1024;
                dt[m * 1024] = df.x;
                dt[plane + m * 1024] = df.y;
                cur[m * n + q] = nv;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// per-step taps: plane sums (ref :7005-7190), phase-centre sample
// (ref :8259-8290).  One block; plane sums reduce in a fixed tree order.
template <typename T>
__global__ void __launch_bounds__(1024, 1) k_taps(const __grid_constant__ AemParams P, const __grid_constant__ TapDev D,
                       const __grid_constant__ FarFieldDev F, int counter, int steps) {
    counter = step_of(P, counter);
    __shared__ T red[4][1024];
    const int tid = threadIdx.x;
    if (D.plane_sum) {
        const int a = D.axis, b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
        const int nb = F.hi[b] - F.lo[b] + 1, nc = F.hi[c] - F.lo[c] + 1;
        const int i_lo = P.lo[a], i_hi = P.hi[a];
        T acc[4] = {zero<T>(), zero<T>(), zero<T>(), zero<T>()};
        // a thread's points q = tid, tid + B, tid + 2B, ... in that order;
        // the loads of four points are issued before their sums
        constexpr int QU = 4;
        const int nq = nb * nc;
        for (int q0 = tid; q0 < nq; q0 += QU * blockDim.x) {
            T ev[QU][2][2];
#pragma unroll
            for (int u = 0; u < QU; u++) {
                const int q = q0 + u * blockDim.x;
                if (q >= nq) continue;
                int idx[3];
                idx[b] = F.lo[b] + q % nb;
                idx[c] = F.lo[c] + q / nb;
                for (int side = 0; side < 2; side++) {
                    idx[a] = side ? i_hi : i_lo;
                    // the two transverse components: x plane (Ez, Ey), y (Ez, Ex), z (Ey, Ex)
                    ev[u][side][0] = fget<T>(P, P.E[a == 2 ? 1 : 2], idx[0], idx[1], idx[2]);
                    ev[u][side][1] = fget<T>(P, P.E[a == 0 ? 1 : 0], idx[0], idx[1], idx[2]);
                }
            }
#pragma unroll
            for (int u = 0; u < QU; u++) {
            if (q0 + u * (int)blockDim.x >= nq) continue;
            for (int side = 0; side < 2; side++) {
                const T e1 = ev[u][side][0], e2 = ev[u][side][1];
                if (!P.kmax) {
                    T v;
                    if (a == 0) v = e1 * D.w1 - e2 * D.w2;
                    else v = e1 * D.w1 + e2 * D.w2;
                    acc[side] = acc[side] + v;
                } else {
                    // TE / TM projections with k_num_*_exception, ref :7122-7177
                    const float ku = D.knum[a == 0 ? 1 : 0], kv = D.knum[a == 2 ? 1 : 2];
                    T te, tm;
                    if (a == 2) { te = e2 * D.knum[1] - e1 * D.knum[0]; tm = e2 * D.knum[0] + e1 * D.knum[1]; }
                    else { te = e1 * ku - e2 * kv; tm = e1 * kv + e2 * ku; }
                    acc[side] = acc[side] + te;
                    acc[2 + side] = acc[2 + side] + tm;
                }
            }
            }
        }
        for (int m = 0; m < 4; m++) red[m][tid] = acc[m];
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if (tid < w)
                for (int m = 0; m < 4; m++) red[m][tid] = red[m][tid] + red[m][tid + w];
            __syncthreads();
        }
        if (tid == 0) {
            at<T>(D.refl, counter - 1) = at<T>(D.refl, counter - 1) + red[0][0];
            at<T>(D.trans, counter - 1) = at<T>(D.trans, counter - 1) + red[1][0];
            if (P.kmax) {
                at<T>(D.refl_tm, counter - 1) = at<T>(D.refl_tm, counter - 1) + red[2][0];
                at<T>(D.trans_tm, counter - 1) = at<T>(D.trans_tm, counter - 1) + red[3][0];
            }
        }
    }
    if (D.ff_pc && tid == 0) {
        const int i = D.ic, j = D.jc, k = D.kc;
        const void *Ex = P.E[0], *Ey = P.E[1], *Ez = P.E[2], *Hx = P.H[0], *Hy = P.H[1], *Hz = P.H[2];
        at<T>(D.pc[0], counter - 1) = (fget<T>(P, Ex, i, j, k) + fget<T>(P, Ex, i, j + 1, k) + fget<T>(P, Ex, i, j, k + 1) + fget<T>(P, Ex, i, j + 1, k + 1)) / 4.0f;
        at<T>(D.pc[1], counter - 1) = (fget<T>(P, Ey, i, j, k) + fget<T>(P, Ey, i + 1, j, k) + fget<T>(P, Ey, i, j, k + 1) + fget<T>(P, Ey, i + 1, j, k + 1)) / 4.0f;
        at<T>(D.pc[2], counter - 1) = (fget<T>(P, Ez, i, j, k) + fget<T>(P, Ez, i + 1, j, k) + fget<T>(P, Ez, i, j + 1, k) + fget<T>(P, Ez, i + 1, j + 1, k)) / 4.0f;
        const T hx = (fget<T>(P, Hx, i, j, k) + fget<T>(P, Hx, i + 1, j, k)) / 4.0f;
        const T hy = (fget<T>(P, Hy, i, j, k) + fget<T>(P, Hy, i, j + 1, k)) / 4.0f;
        const T hz = (fget<T>(P, Hz, i, j, k) + fget<T>(P, Hz, i, j, k + 1)) / 4.0f;
        at<T>(D.pc[3], counter - 1) = hx; at<T>(D.pc[4], counter - 1) = hy; at<T>(D.pc[5], counter - 1) = hz;
        if (counter < steps) { at<T>(D.pc[3], counter) = hx; at<T>(D.pc[4], counter) = hy; at<T>(D.pc[5], counter) = hz; }
    }
    if (tid < 3 * D.nprobe) {
        // point probes: cell-centred E as the phase-centre sample (ref :8273-8275)
        const int pq = tid / 3, c = tid % 3;
        const int i = D.prb_idx[pq][0], j = D.prb_idx[pq][1], k = D.prb_idx[pq][2];
        T v;
        if (c == 0) v = (fget<T>(P, P.E[0], i, j, k) + fget<T>(P, P.E[0], i, j + 1, k) + fget<T>(P, P.E[0], i, j, k + 1) + fget<T>(P, P.E[0], i, j + 1, k + 1)) / 4.0f;
        else if (c == 1) v = (fget<T>(P, P.E[1], i, j, k) + fget<T>(P, P.E[1], i + 1, j, k) + fget<T>(P, P.E[1], i, j, k + 1) + fget<T>(P, P.E[1], i + 1, j, k + 1)) / 4.0f;
        else v = (fget<T>(P, P.E[2], i, j, k) + fget<T>(P, P.E[2], i + 1, j, k) + fget<T>(P, P.E[2], i, j + 1, k) + fget<T>(P, P.E[2], i + 1, j + 1, k)) / 4.0f;
        at<T>(D.prb, (long long)tid * steps + counter - 1) = v;
    }
    if (D.ndft) {
        // this step's samples are in place (plane sums above, port voltages
        // from the E half-step's port kernel)
        __syncthreads();
        const long long m = counter - 1;
        for (int q = tid; q < D.nser * D.ndft; q += blockDim.x) {
            const int sr = q / D.ndft, f = q % D.ndft;
            const T x = at<T>(const_cast<void*>(D.ser[sr]), m);
            double xr, xi;
            if constexpr (sizeof(T) == sizeof(float)) { xr = (double)x; xi = 0.0; }
            else { xr = (double)x.x; xi = (double)x.y; }
            // phase in half-turns, reduced to [0, 2) before sincospi
            double ph = (2.0 * D.dft_f[f] * D.dft_dt) * (double)m;
            ph -= 2.0 * floor(0.5 * ph);
            double sn, cs;
            sincospi(ph, &sn, &cs);
            // (xr + i xi)(cs - i sn), added with Kahan compensation
            const double tr = xr * cs + xi * sn, ti = xi * cs - xr * sn;
            double* acc = D.dft_acc + 2 * (long long)q;
            double* cmp = D.dft_cmp + 2 * (long long)q;
            const double yr = tr - cmp[0], sr_ = acc[0] + yr;
            cmp[0] = (sr_ - acc[0]) - yr;
            acc[0] = sr_;
            const double yi = ti - cmp[1], si = acc[1] + yi;
            cmp[1] = (si - acc[1]) - yi;
            acc[1] = si;
        }
    }
}

// watchdog: flag a non-finite value (exponent bits all set) in any of the
// six field arrays, read as float4 (n4 float4 per array)
__global__ void k_nonfinite(const __grid_constant__ FieldPtrs F, long long n4, int* flag) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    bool bad = false;
    for (int a = 0; a < 6; a++) {
        const uint4* p = reinterpret_cast<const uint4*>(F.p[a]);
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
            const uint4 v = __ldg(p + i);
            bad |= ((v.x & 0x7f800000u) == 0x7f800000u) | ((v.y & 0x7f800000u) == 0x7f800000u) |
                   ((v.z & 0x7f800000u) == 0x7f800000u) | ((v.w & 0x7f800000u) == 0x7f800000u);
        }
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicExch(flag, 1);
}

int launch_nonfinite(const FieldPtrs& F, long long n4, int* flag, cudaStream_t s) {
    k_nonfinite<<<148 * 4, 256, 0, s>>>(F, n4, flag);
    return 1;
}

// 2-D video slice, ref :6833-6958 (cell-centred E, H halves at both steps)
template <typename T>
__global__ void k_video(const __grid_constant__ AemParams P, const __grid_constant__ TapDev D, int counter, int steps) {
    counter = step_of(P, counter);
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= D.v1 * D.v2) return;
    const int va = q % D.v1 + 1, vb = q / D.v1 + 1;
    int i, j, k;
    if (D.slice_dir == 0) { i = D.slice_loc; j = va; k = vb; }
    else if (D.slice_dir == 1) { i = va; j = D.slice_loc; k = vb; }
    else { i = va; j = vb; k = D.slice_loc; }
    const void *Ex = P.E[0], *Ey = P.E[1], *Ez = P.E[2], *Hx = P.H[0], *Hy = P.H[1], *Hz = P.H[2];
    const long long o = ((long long)(counter - 1) * D.v2 + (vb - 1)) * D.v1 + (va - 1);
    const long long o1 = o + (long long)D.v1 * D.v2;
    at<T>(D.vid[0], o) = (fget<T>(P, Ex, i, j, k) + fget<T>(P, Ex, i, j + 1, k) + fget<T>(P, Ex, i, j, k + 1) + fget<T>(P, Ex, i, j + 1, k + 1)) / 4.0f;
    at<T>(D.vid[2], o) = (fget<T>(P, Ey, i, j, k) + fget<T>(P, Ey, i + 1, j, k) + fget<T>(P, Ey, i, j, k + 1) + fget<T>(P, Ey, i + 1, j, k + 1)) / 4.0f;
    at<T>(D.vid[4], o) = (fget<T>(P, Ez, i, j, k) + fget<T>(P, Ez, i + 1, j, k) + fget<T>(P, Ez, i, j + 1, k) + fget<T>(P, Ez, i + 1, j + 1, k)) / 4.0f;
    const T hx = (fget<T>(P, Hx, i, j, k) + fget<T>(P, Hx, i + 1, j, k)) / 4.0f;
    const T hy = (fget<T>(P, Hy, i, j, k) + fget<T>(P, Hy, i, j + 1, k)) / 4.0f;
    const T hz = (fget<T>(P, Hz, i, j, k) + fget<T>(P, Hz, i, j, k + 1)) / 4.0f;
    at<T>(D.vid[1], o) = hx; at<T>(D.vid[3], o) = hy; at<T>(D.vid[5], o) = hz;
    if (counter < steps) { at<T>(D.vid[1], o1) = hx; at<T>(D.vid[3], o1) = hy; at<T>(D.vid[5], o1) = hz; }
}

// Full-field export, ref :6960-7003: cell-centred averages of all six
// components over i = 1..X-1-pbc_x, j = 1..Y-1-pbc_y, k = 1..Z-1-pbc_z (E at
// the step, H half a step earlier, as the reference writes them), stored
// component-major, i fastest: out[comp][k][j][i] in the reference's order
// Ex, Ey, Ez, Hx, Hy, Hz.  Sums left to right as in the Fortran expression;
// the divisions by 4 and 2 are exact.
template <typename T>
__global__ void k_full(const __grid_constant__ AemParams P, void* out, int n1, int n2, int n3) {
    const long long n = (long long)n1 * n2 * n3;
    const void *Ex = P.E[0], *Ey = P.E[1], *Ez = P.E[2], *Hx = P.H[0], *Hy = P.H[1], *Hz = P.H[2];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % n1) + 1, j = (int)((q / n1) % n2) + 1, k = (int)(q / ((long long)n1 * n2)) + 1;
        at<T>(out, q) = (fget<T>(P, Ex, i, j, k) + fget<T>(P, Ex, i, j + 1, k) + fget<T>(P, Ex, i, j, k + 1) + fget<T>(P, Ex, i, j + 1, k + 1)) / 4.0f;
        at<T>(out, q + n) = (fget<T>(P, Ey, i, j, k) + fget<T>(P, Ey, i + 1, j, k) + fget<T>(P, Ey, i, j, k + 1) + fget<T>(P, Ey, i + 1, j, k + 1)) / 4.0f;
        at<T>(out, q + 2 * n) = (fget<T>(P, Ez, i, j, k) + fget<T>(P, Ez, i + 1, j, k) + fget<T>(P, Ez, i, j + 1, k) + fget<T>(P, Ez, i + 1, j + 1, k)) / 4.0f;
        at<T>(out, q + 3 * n) = (fget<T>(P, Hx, i, j, k) + fget<T>(P, Hx, i + 1, j, k)) / 2.0f;
        at<T>(out, q + 4 * n) = (fget<T>(P, Hy, i, j, k) + fget<T>(P, Hy, i, j + 1, k)) / 2.0f;
        at<T>(out, q + 5 * n) = (fget<T>(P, Hz, i, j, k) + fget<T>(P, Hz, i, j, k + 1)) / 2.0f;
    }
}

int launch_full(const AemParams& P, void* out, const int n[3], cudaStream_t s) {
    const long long cells = (long long)n[0] * n[1] * n[2];
    if (cells <= 0) return 0;
    const int blocks = (int)((cells + 255) / 256 < 148 * 8 ? (cells + 255) / 256 : 148 * 8);
    if (P.kmax) k_full<cf><<<blocks, 256, 0, s>>>(P, out, n[0], n[1], n[2]);
    else k_full<float><<<blocks, 256, 0, s>>>(P, out, n[0], n[1], n[2]);
    return 1;
}

// ---------------------------------------------------------------------------
// graph replay: the step counter advances once at the end of every step
__global__ void k_step_advance(int* d) { *d += 1; }
int launch_step_advance(int* d, cudaStream_t s) {
    k_step_advance<<<1, 1, 0, s>>>(d);
    return 1;
}

int launch_ports_h(const AemParams& P, const PortSet& ps, int counter, cudaStream_t s) {
    if (!ps.n) return 0;
    if (P.kmax) k_ports_h<cf><<<1, 512, 0, s>>>(P, ps, counter);
    else k_ports_h<float><<<1, 512, 0, s>>>(P, ps, counter);
    return 1;
}
int launch_ports_e(const AemParams& P, const PortSet& ps, int counter, cudaStream_t s) {
    if (!ps.n) return 0;
    if (P.kmax) k_ports_e<cf><<<1, 512, 0, s>>>(P, ps, counter);
    else k_ports_e<float><<<1, 512, 0, s>>>(P, ps, counter);
    return 1;
}
int launch_ff_currents(const AemParams& P, const FarFieldDev& F, int slot, cudaStream_t s) {
    if (!F.nang) return 0;
    long long tot = 2 * (F.face_n[0] + F.face_n[1] + F.face_n[2]);
    if (tot == 0) return 0;
    int blocks = (int)((tot + 255) / 256 < 148 * 16 ? (tot + 255) / 256 : 148 * 16);
    if (P.kmax) k_ff_currents<cf><<<blocks, 256, 0, s>>>(P, F, slot);
    else k_ff_currents<float><<<blocks, 256, 0, s>>>(P, F, slot);
    return 1;
}
int launch_taps(const AemParams& P, const TapDev& D, const FarFieldDev& F, int counter, int steps, cudaStream_t s) {
    int n = 0;
    if (D.plane_sum || D.ff_pc || D.ndft || D.nprobe) {
        if (P.kmax) k_taps<cf><<<1, 1024, 0, s>>>(P, D, F, counter, steps);
        else k_taps<float><<<1, 1024, 0, s>>>(P, D, F, counter, steps);
        n++;
    }
    if (D.video) {
        int cells = D.v1 * D.v2;
        if (P.kmax) k_video<cf><<<(cells + 255) / 256, 256, 0, s>>>(P, D, counter, steps);
        else k_video<float><<<(cells + 255) / 256, 256, 0, s>>>(P, D, counter, steps);
        n++;
    }
    return n;
}

}  // namespace aem
