// aem_dev.cuh -- device helpers shared by the B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "aem_types.h"

namespace aem {

// complex FP32 field value (kmax solver); the standard solver uses float
struct cf {
    float x, y;
};
__host__ __device__ inline cf operator+(cf a, cf b) { return {a.x + b.x, a.y + b.y}; }
__host__ __device__ inline cf operator-(cf a, cf b) { return {a.x - b.x, a.y - b.y}; }
__host__ __device__ inline cf operator*(float s, cf a) { return {s * a.x, s * a.y}; }
__host__ __device__ inline cf operator*(cf a, float s) { return {a.x * s, a.y * s}; }
__host__ __device__ inline cf operator/(cf a, float s) { return {a.x / s, a.y / s}; }
__host__ __device__ inline cf cmul(cf a, cf b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }

template <typename T> __device__ inline T zero();
template <> __device__ inline float zero<float>() { return 0.0f; }
template <> __device__ inline cf zero<cf>() { return {0.0f, 0.0f}; }

// multiply by exp(sign * i k L) along axis a (kmax Bloch phase); identity
// for real fields
template <typename T> __device__ inline T bloch(T v, const AemParams& P, int a, int sign);
template <> __device__ inline float bloch<float>(float v, const AemParams&, int, int) { return v; }
template <> __device__ inline cf bloch<cf>(cf v, const AemParams& P, int a, int sign) {
    cf ph = {P.bloch_re[a], sign > 0 ? P.bloch_im[a] : -P.bloch_im[a]};
    return cmul(v, ph);
}

// Reference index that a storage position stands for when testing the
// reference's loop bounds.  On a periodic axis position 0 is index 1 for H
// and for the normal E component, but for a tangential E component the
// surviving value is the one the reference computed at index N-1 (its PBC
// step copies N-1 onto 1, fdtd_solver.f90:6672-6741).
__device__ inline int rep_idx(const AemParams& P, int a, int p, bool tangential_e) {
    if (P.per[a] && p == 0 && tangential_e) return (a == 0 ? P.X : a == 1 ? P.Y : P.Z) - 1;
    return p + 1;
}

__device__ inline int wrap_up(const AemParams& P, int a, int p, int S, bool* wrapped) {
    *wrapped = false;
    if (p + 1 == S && P.per[a]) { *wrapped = true; return 0; }
    return p + 1;
}
__device__ inline int wrap_dn(const AemParams& P, int a, int p, int S, bool* wrapped) {
    *wrapped = false;
    if (p == 0 && P.per[a]) { *wrapped = true; return S - 1; }
    return p - 1;
}

// num / dl of the CPML update psi = b psi + c diff / dl (num = c diff),
// rounded as written.  A zero numerator is returned as it is: +-0 / dl
// (dl > 0) is that same signed zero, and the IEEE division would otherwise
// take its slow path for it (the CPML fields are exactly zero until a wave
// reaches them).  The test is a real branch (a select would still run the
// division); the division is the one `/` compiles to with -ftz=true.
__device__ __forceinline__ float cpml_div(float num, float dl) {
    float q;
    asm("{\n\t.reg .pred z;\n\tmov.b32 %0, %1;\n\tsetp.eq.f32 z, %1, 0f00000000;\n\t@z bra CPML_DIV_DONE;\n\t"
        "div.rn.ftz.f32 %0, %1, %2;\n\tCPML_DIV_DONE:\n\t}"
        : "=f"(q)
        : "f"(num), "f"(dl));
    return q;
}
__device__ __forceinline__ cf cpml_div(cf num, float dl) { return {cpml_div(num.x, dl), cpml_div(num.y, dl)}; }

// Per-block copies of the small tables the volume kernels index per cell:
// uniform-edge Ga/Gb and cell eps/sigma per material, CPML b/c per slab
// depth.  Shared memory keeps the id -> coefficient lookup off the global
// memory latency chain and serves lanes at different CPML depths in one
// access (the same values, so results are unchanged).
struct CoefTabs {
    float ga[AEM_MAX_MATERIALS][3], gb[AEM_MAX_MATERIALS][3];
    float eps[AEM_MAX_MATERIALS][3], sig[AEM_MAX_MATERIALS][3];
    float be[3][2][AEM_MAX_PML], ce[3][2][AEM_MAX_PML], bh[3][2][AEM_MAX_PML], ch[3][2][AEM_MAX_PML];
};

// fill the block's tables; every thread of the block must call it (it ends
// with a barrier), before any thread leaves the kernel
__device__ inline void load_coef_tabs(const AemParams& P, CoefTabs& T) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (int q = tid; q < P.nmat * 3; q += nt) {
        const int m = q / 3, c = q % 3;
        T.ga[m][c] = P.ucoef[m].ga[c];
        T.gb[m][c] = P.ucoef[m].gb[c];
        T.eps[m][c] = P.mat[m].eps[c];
        T.sig[m][c] = P.mat[m].sig[c];
    }
    for (int q = tid; q < 3 * 2 * AEM_MAX_PML; q += nt) {
        const int a = q / (2 * AEM_MAX_PML), sd = (q / AEM_MAX_PML) % 2, d = q % AEM_MAX_PML;
        if (d >= P.npml[a][sd]) continue;
        T.be[a][sd][d] = P.be[a][sd][d];
        T.ce[a][sd][d] = P.ce[a][sd][d];
        T.bh[a][sd][d] = P.bh[a][sd][d];
        T.ch[a][sd][d] = P.ch[a][sd][d];
    }
    __syncthreads();
}

// the step number of this launch: the device counter during graph replay,
// else the launch argument
__device__ __forceinline__ int step_of(const AemParams& P, int counter) { return P.dstep ? *P.dstep : counter; }

__device__ inline long long lin(const AemParams& P, int px, int py, int pz) {
    return ((long long)pz * P.SY + py) * P.PX + px;
}

// storage index of a CPML psi value: slab axis a, depth q (1-based)
__device__ inline long long psi_idx(const AemParams& P, int a, int q, int px, int py, int pz, int n) {
    int c0 = a == 0 ? q - 1 : px, c1 = a == 1 ? q - 1 : py, c2 = a == 2 ? q - 1 : pz;
    int e0 = a == 0 ? n : P.PX, e1 = a == 1 ? n : P.SY;
    return ((long long)c2 * e1 + c1) * e0 + c0;
}

// Ga/Gb of the reference (:2837-2853) and Drude Ja/Jb (:2870-2875)
__device__ inline float d_ga(float s, float e, float dt) {
    const float ep0 = 8.85418782E-12f;
    return __fdiv_rn(1.0f - __fdiv_rn(s * dt, 2.0f * ep0 * e), 1.0f + __fdiv_rn(s * dt, 2.0f * ep0 * e));
}
__device__ inline float d_gb(float s, float e, float dt) {
    const float ep0 = 8.85418782E-12f;
    return __fdiv_rn(__fdiv_rn(dt, ep0 * e), 1.0f + __fdiv_rn(s * dt, 2.0f * ep0 * e));
}
__device__ inline float d_ja(float g, float dt) {
    return __fdiv_rn(1.0f - g * dt / 2.0f, 1.0f + g * dt / 2.0f);
}
__device__ inline float d_jb(float w, float g, float dt) {
    const double ep0 = (double)8.85418782E-12f;
    return (float)(((double)w * (double)w * ep0 * (double)dt / 2.0) / (double)(1.0f + g * dt / 2.0f));
}

// Incident plane-wave function Inc of the standard solver, ref :8825-8842
__device__ inline float d_inc(const AemParams& P, int m, float w, float x, float y, float z, float cnt) {
    float tx = P.sc[m][0] * (x - (float)P.delay[m][0]) * P.del[0];
    float ty = P.sc[m][1] * (y - (float)P.delay[m][1]) * P.del[1];
    float tz = P.sc[m][2] * (z - (float)P.delay[m][2]) * P.del[2];
    float arg = __fdiv_rn(P.t_spread - (cnt * P.dt) + P.inv_c * (tx + ty + tz), P.spread);
    if (P.pulse_type == 1) return w * expf(-0.5f * (arg * arg));
    if (P.pulse_type == 2) return -1.0f * w * arg * P.exp_half * expf(-0.5f * (arg * arg));
    return 0.0f;
}

// kmax plane source Inc, ref :8861-8887: real envelope times Bloch phase
__device__ inline cf d_inc_k(const AemParams& P, float w, float xf, float ku, float du, float kv, float dv, float cnt,
                             float dxf) {
    float a = __fdiv_rn(P.t_spread - (cnt * P.dt) + P.inv_c * (xf * dxf), P.spread);
    float env = w * expf(-0.5f * (a * a));
    float ph = P.two_pi_f * ((cnt * P.dt) + P.inv_c * (xf * dxf)) - (ku * du + kv * dv);
    float s, c;
    sincosf(ph, &s, &c);
    return {env * c, env * s};
}

}  // namespace aem
