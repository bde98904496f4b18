// aem_yee4.cu -- fused H+E step, 4 cells per thread, tiles fed by TMA
// (grids without x/y periodicity; any z).
//
// Same arithmetic, statement for statement, as k_update_h / k_update_e
// (bulk curl fdtd_solver.f90:4442-4484 / :5667-5710, CPML :5227-5375 /
// :6522-6670), so the fields are bit-identical to the other paths: every
// FP32 operation of a cell is the reference's, in its order, rounded to
// nearest with subnormals flushed.  (Packed .f32x2 arithmetic is not used:
// the assembler fuses a packed multiply into a following packed add even
// with .rn and contraction disabled, which changes the rounding.)
//
// A CTA owns a 128 x 15 (x, y) column tile and marches a z chunk of 64
// planes.  Warps 0..14 own rows y0..y0+14; lane l owns the four cells
// x0+4l .. x0+4l+3, so every shared-memory and global access of a cell
// group is one 16-byte operation.  Warp 15 computes Hx, Hz of the -y halo
// row (y0-1), which the E update of row y0 needs, and, while the others
// update E, Hy, Hz of the -x halo cells (x0-1) of the next plane.
//
// Per plane p one thread requests by TMA (cp.async.bulk.tensor, zero fill
// outside the grid) E_old(p) on rows y0-1..y0+15, x0-4..x0+131; H_old(p) on
// rows y0-1..y0+14, x0-4..x0+127; the material ids of rows y0-1..y0+14,
// x0-16..x0+127.  Stage t (E(t+1), H(t), ids(t)) completes on its own
// mbarrier; it is requested two planes ahead, while plane t-2 is computed,
// into rings of 4 E planes, 3 H planes and 4 id planes.  One CTA per SM
// (about 217 KB of shared memory).  Fields and H-psi are double-buffered
// (read E/H/psi_h, write E2/H2/psi_h2), so halo values recomputed here
// never race with their owners' stores.
//
// A cell group takes the fast path when its four cells are all
// updated; its CPML terms then follow per slab (x: per cell; y: per row;
// z: per plane; y and z psi as 16-byte accesses).  The E fast path also
// needs the seven surrounding cells to share one material (ga/gb from a
// shared-memory copy of the material table).  Every other cell takes the
// per-cell path with the reference's 4-cell material average.
//
// Waits on the mbarriers give up after 2 s of wall time: the CTA then adds
// to the error counter P.err and returns (the host reports it).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdlib>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "aem_dev.cuh"
#include "aem_kernels.h"

namespace aem {

// 15 owned rows + the -y halo row: 16 warps (512 threads) of at most 128
// registers, one CTA per SM; the warps hide each other's latency
constexpr int Y4_TX = 128, Y4_TY = 15, Y4_ZC = 64, Y4_NT = 32 * (Y4_TY + 1);
constexpr int Y4_EW = Y4_TX + 8, Y4_ER = Y4_TY + 2;   // E box 136 x 17, x from x0-4, y from y0-1
constexpr int Y4_HW = Y4_TX + 4, Y4_HR = Y4_TY + 1;   // H box 132 x 16
constexpr int Y4_IW = Y4_TX + 16, Y4_IR = Y4_TY + 1;  // id box 144 x 16 bytes, x from x0-16
// every TMA destination starts on a 128-byte boundary
constexpr int y4_up128(int b) { return (b + 127) / 128 * 128; }
constexpr int Y4_EC = y4_up128(Y4_ER * Y4_EW * 4) / 4;  // floats from one E component tile to the next
constexpr int Y4_HC = y4_up128(Y4_HR * Y4_HW * 4) / 4;
constexpr int Y4_IC = y4_up128(Y4_IR * Y4_IW);          // bytes from one id tile to the next
// copies run Y4_LA planes ahead: stage t (E(t+1), H(t), ids(t)) is requested
// at plane t-Y4_LA and consumed at plane t; ring depths in planes follow
constexpr int Y4_LA = 2;
constexpr int Y4_ES = Y4_LA + 2, Y4_HS = Y4_LA + 1, Y4_IS = Y4_LA + 2, Y4_NB = Y4_LA + 1;
constexpr int Y4_OFF_H = Y4_ES * 3 * Y4_EC * 4;
constexpr int Y4_OFF_I = Y4_OFF_H + Y4_HS * 3 * Y4_HC * 4;
constexpr int Y4_OFF_HN = Y4_OFF_I + Y4_IS * Y4_IC;
constexpr int Y4_HN_F = 2 * Y4_HR * Y4_TX;  // H_new hx, hz of rows y0-1..y0+14
constexpr int Y4_OFF_DZ = Y4_OFF_HN + Y4_HN_F * 4;
constexpr int Y4_OFF_DX = Y4_OFF_DZ + 2 * Y4_ZC * 4;
constexpr int Y4_OFF_XH = Y4_OFF_DX + (2 * Y4_TX + 4) * 4;
constexpr int Y4_OFF_GAB = Y4_OFF_XH + 2 * Y4_TY * 2 * 4;
constexpr int Y4_OFF_BAR = Y4_OFF_GAB + AEM_MAX_MATERIALS * 6 * 4;
constexpr int Y4_SMEM = Y4_OFF_BAR + Y4_NB * 8;
constexpr unsigned Y4_TX_E = Y4_ER * Y4_EW * 4, Y4_TX_H = Y4_HR * Y4_HW * 4, Y4_TX_I = Y4_IR * Y4_IW;
constexpr unsigned Y4_TX_STAGE = 3 * Y4_TX_E + 3 * Y4_TX_H + Y4_TX_I;          // E(t+1), H(t), ids(t)
constexpr unsigned Y4_TX_FIRST = 9 * Y4_TX_E + 6 * Y4_TX_H + 2 * Y4_TX_I;      // E(z0-1..z0+1), H, ids(z0-1..z0)
static_assert(Y4_OFF_H % 128 == 0 && Y4_OFF_I % 128 == 0 && Y4_OFF_HN % 128 == 0 && Y4_OFF_BAR % 8 == 0, "layout");
static_assert(Y4_TX_FIRST < (1u << 20), "mbarrier transaction count");
static_assert(Y4_SMEM <= 227 * 1024, "shared memory per CTA");

// tensor maps of the current read buffers (3-D: x = pitch PX, y = SY, z = SZ)
struct Y4Maps {
    CUtensorMap e[3], h[3], id;
};

// ---- shared memory, mbarriers and TMA ----
__device__ __forceinline__ unsigned y4_sa(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void y4_bar_init(uint64_t* b) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(y4_sa(b)) : "memory");
}
__device__ __forceinline__ void y4_bar_expect(uint64_t* b, unsigned tx) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(y4_sa(b)), "r"(tx) : "memory");
}
__device__ __forceinline__ bool y4_bar_try(uint64_t* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(y4_sa(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long y4_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// wait for phase `parity` of barrier b; false after 2 s of wall time
__device__ __forceinline__ bool y4_bar_wait(uint64_t* b, unsigned parity) {
    if (y4_bar_try(b, parity)) return true;
    const unsigned long long t0 = y4_ns();
    while (!y4_bar_try(b, parity))
        if (y4_ns() - t0 > 2000000000ull) return false;
    return true;
}
// one box of plane z (z outside 0..SZ-1: zero fill) at (x, y) into dst
__device__ __forceinline__ void y4_tma(void* dst, const CUtensorMap* m, int x, int y, int z, uint64_t* b) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(y4_sa(dst)),
        "l"(m), "r"(x), "r"(y), "r"(z), "r"(y4_sa(b))
        : "memory");
}

__device__ inline float ldf4(const void* b, long long i) { return reinterpret_cast<const float*>(b)[i]; }
__device__ inline void stf4(void* b, long long i, float v) { reinterpret_cast<float*>(b)[i] = v; }

__device__ inline float psi4(const void* rd, void* wr, bool store, float b, float c, float diff, float dl, long long q) {
    const float nw = b * ldf4(rd, q) + cpml_div(c * diff, dl);
    if (store) stf4(wr, q, nw);
    return nw;
}

// store the cells of mask mk of 4 consecutive floats at base + q
__device__ __forceinline__ void y4_store4_f(void* base, long long q, unsigned mk, const float v[4]) {
    float* w = reinterpret_cast<float*>(base) + q;
    if (mk == 0xFu) {
        *reinterpret_cast<float4*>(w) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int e = 0; e < 4; e++)
            if (mk >> e & 1u) w[e] = v[e];
    }
}

// two CPML terms of one slab over four x-contiguous cells (same depth q,
// same b, c): both psi rows are loaded before either is used, so the two
// loads overlap (the arrays may alias as far as the compiler knows)
__device__ __forceinline__ void y4_psi_row2(const void* rdA, void* wrA, unsigned mkA, const float dA[4], float gA,
                                            float fA[4], const void* rdB, void* wrB, unsigned mkB, const float dB[4],
                                            float gB, float fB[4], bool store, float b, float c, float dl, long long q) {
    const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float4 oA = mkA ? *reinterpret_cast<const float4*>(reinterpret_cast<const float*>(rdA) + q) : z4;
    const float4 oB = mkB ? *reinterpret_cast<const float4*>(reinterpret_cast<const float*>(rdB) + q) : z4;
    const float va[4] = {oA.x, oA.y, oA.z, oA.w}, vb[4] = {oB.x, oB.y, oB.z, oB.w};
    float na[4], nb[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        na[e] = b * va[e] + cpml_div(c * dA[e], dl);
        nb[e] = b * vb[e] + cpml_div(c * dB[e], dl);
    }
    if (mkA) {
#pragma unroll
        for (int e = 0; e < 4; e++) fA[e] = fA[e] + gA * na[e];
    }
    if (mkB) {
#pragma unroll
        for (int e = 0; e < 4; e++) fB[e] = fB[e] + gB * nb[e];
    }
    if (!store) return;
    if (mkA) y4_store4_f(wrA, q, mkA, na);
    if (mkB) y4_store4_f(wrB, q, mkB, nb);
}

// store the cells of mask mk of a 4-cell group (16 bytes when all four)
__device__ __forceinline__ void y4_store4(void* base, long long c, unsigned mk, const float v[4]) {
    float* w = reinterpret_cast<float*>(base) + c;
    if (mk == 0xFu) {
        *reinterpret_cast<float4*>(w) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int e = 0; e < 4; e++)
            if (mk >> e & 1u) w[e] = v[e];
    }
}

// H_new of one cell (k_update_h's expressions; psi from psi_h, to psi_h2 when store)
__device__ __forceinline__ float3 y4_h_cell(const AemParams& P, int px, int py, int pz, float ex, float ey, float ez,
                                          float ex_jp, float ez_jp, float ey_ip, float ez_ip, float ex_kp, float ey_kp,
                                          float hx0, float hy0, float hz0, bool store) {
    const int i = px + 1, j = py + 1, k = pz + 1;
    const float DB = P.DB;
    const float dhx = P.den_h[0][i - 1], dhy = P.den_h[1][j - 1], dhz = P.den_h[2][k - 1];
    float hxv = hx0 + DB * ((ez - ez_jp) * dhy + (ey_kp - ey) * dhz);
    float hyv = hy0 + DB * ((ez_ip - ez) * dhx + (ex - ex_kp) * dhz);
    float hzv = hz0 + DB * ((ey - ey_ip) * dhx + (ex_jp - ex) * dhy);
    const int qx_lo = (i <= P.npml[0][0] - 1) ? i : 0, qx_hi = (i >= P.X + 1 - P.npml[0][1]) ? P.X - i : 0;
    const int qy_lo = (j <= P.npml[1][0] - 1) ? j : 0, qy_hi = (j >= P.Y + 1 - P.npml[1][1]) ? P.Y - j : 0;
    const int qz_lo = (k <= P.npml[2][0] - 1) ? k : 0, qz_hi = (k >= P.Z + 1 - P.npml[2][1]) ? P.Z - k : 0;
    if (!(qx_lo | qx_hi | qy_lo | qy_hi | qz_lo | qz_hi)) return make_float3(hxv, hyv, hzv);
    if (qy_lo) hxv = hxv + DB * psi4(P.psi_h[0][1][0], P.psi_h2[0][1][0], store, P.bh[1][0][qy_lo - 1], P.ch[1][0][qy_lo - 1], ez - ez_jp, P.del[1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]));
    if (qy_hi) hxv = hxv + DB * psi4(P.psi_h[0][1][1], P.psi_h2[0][1][1], store, P.bh[1][1][qy_hi - 1], P.ch[1][1][qy_hi - 1], ez - ez_jp, P.del[1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]));
    if (qz_lo) hxv = hxv + DB * psi4(P.psi_h[0][2][0], P.psi_h2[0][2][0], store, P.bh[2][0][qz_lo - 1], P.ch[2][0][qz_lo - 1], ey_kp - ey, P.del[2], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]));
    if (qz_hi) hxv = hxv + DB * psi4(P.psi_h[0][2][1], P.psi_h2[0][2][1], store, P.bh[2][1][qz_hi - 1], P.ch[2][1][qz_hi - 1], ey_kp - ey, P.del[2], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]));
    if (qx_lo) hyv = hyv + DB * psi4(P.psi_h[1][0][0], P.psi_h2[1][0][0], store, P.bh[0][0][qx_lo - 1], P.ch[0][0][qx_lo - 1], ez_ip - ez, P.del[0], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]));
    if (qx_hi) hyv = hyv + DB * psi4(P.psi_h[1][0][1], P.psi_h2[1][0][1], store, P.bh[0][1][qx_hi - 1], P.ch[0][1][qx_hi - 1], ez_ip - ez, P.del[0], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]));
    if (qz_lo) hyv = hyv + DB * psi4(P.psi_h[1][2][0], P.psi_h2[1][2][0], store, P.bh[2][0][qz_lo - 1], P.ch[2][0][qz_lo - 1], ex - ex_kp, P.del[2], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]));
    if (qz_hi) hyv = hyv + DB * psi4(P.psi_h[1][2][1], P.psi_h2[1][2][1], store, P.bh[2][1][qz_hi - 1], P.ch[2][1][qz_hi - 1], ex - ex_kp, P.del[2], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]));
    if (qx_lo) hzv = hzv + DB * psi4(P.psi_h[2][0][0], P.psi_h2[2][0][0], store, P.bh[0][0][qx_lo - 1], P.ch[0][0][qx_lo - 1], ey - ey_ip, P.del[0], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]));
    if (qx_hi) hzv = hzv + DB * psi4(P.psi_h[2][0][1], P.psi_h2[2][0][1], store, P.bh[0][1][qx_hi - 1], P.ch[0][1][qx_hi - 1], ey - ey_ip, P.del[0], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]));
    if (qy_lo) hzv = hzv + DB * psi4(P.psi_h[2][1][0], P.psi_h2[2][1][0], store, P.bh[1][0][qy_lo - 1], P.ch[1][0][qy_lo - 1], ex_jp - ex, P.del[1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]));
    if (qy_hi) hzv = hzv + DB * psi4(P.psi_h[2][1][1], P.psi_h2[2][1][1], store, P.bh[1][1][qy_hi - 1], P.ch[1][1][qy_hi - 1], ex_jp - ex, P.del[1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]));
    return make_float3(hxv, hyv, hzv);
}

// x-slab CPML terms of the four cells xb..xb+3 of one H row (Hy, Hz; low
// slab before high slab), added before the y and z terms.  All psi loads are
// issued before any is used.  dzx = ez_ip - ez, dyx = ey - ey_ip; cells
// outside mask mk are left alone.
__device__ __forceinline__ void y4_h_xpml4(const AemParams& P, int xb, int py, int pz, unsigned mk, const float dzx[4],
                                           const float dyx[4], bool store, float hy[4], float hz[4]) {
    const float DB = P.DB;
    int q[2][4];
    long long idx[2][4];
    float oy[2][4], oz[2][4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int i = xb + e + 1;
        q[0][e] = (mk >> e & 1u) && i <= P.npml[0][0] - 1 ? i : 0;
        q[1][e] = (mk >> e & 1u) && i >= P.X + 1 - P.npml[0][1] ? P.X - i : 0;
    }
#pragma unroll
    for (int sd = 0; sd < 2; sd++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            idx[sd][e] = q[sd][e] ? psi_idx(P, 0, q[sd][e], xb + e, py, pz, P.npml[0][sd]) : 0;
            oy[sd][e] = q[sd][e] ? ldf4(P.psi_h[1][0][sd], idx[sd][e]) : 0.0f;
            oz[sd][e] = q[sd][e] ? ldf4(P.psi_h[2][0][sd], idx[sd][e]) : 0.0f;
        }
#pragma unroll
    for (int e = 0; e < 4; e++)
#pragma unroll
        for (int sd = 0; sd < 2; sd++) {
            if (!q[sd][e]) continue;
            const float b = P.bh[0][sd][q[sd][e] - 1], c = P.ch[0][sd][q[sd][e] - 1];
            const float ny = b * oy[sd][e] + cpml_div(c * dzx[e], P.del[0]);
            const float nz = b * oz[sd][e] + cpml_div(c * dyx[e], P.del[0]);
            hy[e] = hy[e] + DB * ny;
            hz[e] = hz[e] + DB * nz;
            if (store) {
                stf4(P.psi_h2[1][0][sd], idx[sd][e], ny);
                stf4(P.psi_h2[2][0][sd], idx[sd][e], nz);
            }
        }
}

// x-slab CPML terms of the four cells of one E row (Ey for the cells of my,
// Ez for those of mz; low slab before high slab), added before the y and z
// terms; all psi loads first.  dzx = hz(i-1) - hz, dyx = hy - hy(i-1).
__device__ __forceinline__ void y4_e_xpml4(const AemParams& P, int xb, int py, int pz, unsigned my, unsigned mz,
                                           const float dzx[4], const float dyx[4], float gby, float gbz, float ey[4],
                                           float ez[4]) {
    int q[2][4];
    long long idx[2][4];
    float oy[2][4], oz[2][4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int i = xb + e + 1;
        const bool any = (my | mz) >> e & 1u;
        q[0][e] = any && i >= 2 && i <= P.npml[0][0] ? i : 0;
        q[1][e] = any && i >= P.X + 1 - P.npml[0][1] && i <= P.X - 1 ? P.X + 1 - i : 0;
    }
#pragma unroll
    for (int sd = 0; sd < 2; sd++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            idx[sd][e] = q[sd][e] ? psi_idx(P, 0, q[sd][e], xb + e, py, pz, P.npml[0][sd]) : 0;
            oy[sd][e] = q[sd][e] && (my >> e & 1u) ? ldf4(P.psi_e[1][0][sd], idx[sd][e]) : 0.0f;
            oz[sd][e] = q[sd][e] && (mz >> e & 1u) ? ldf4(P.psi_e[2][0][sd], idx[sd][e]) : 0.0f;
        }
#pragma unroll
    for (int e = 0; e < 4; e++)
#pragma unroll
        for (int sd = 0; sd < 2; sd++) {
            if (!q[sd][e]) continue;
            const float b = P.be[0][sd][q[sd][e] - 1], c = P.ce[0][sd][q[sd][e] - 1];
            if (my >> e & 1u) {
                const float ny = b * oy[sd][e] + cpml_div(c * dzx[e], P.del[0]);
                ey[e] = ey[e] + gby * ny;
                stf4(P.psi_e[1][0][sd], idx[sd][e], ny);
            }
            if (mz >> e & 1u) {
                const float nz = b * oz[sd][e] + cpml_div(c * dyx[e], P.del[0]);
                ez[e] = ez[e] + gbz * nz;
                stf4(P.psi_e[2][0][sd], idx[sd][e], nz);
            }
        }
}

__device__ inline void y4_gagb(const AemParams& P, const float* gab, int c, int i0, int i1, int i2, int i3, float& ga,
                               float& gb) {
    if (i0 == i1 && i0 == i2 && i0 == i3) {
        ga = gab[i0 * 6 + c];
        gb = gab[i0 * 6 + 3 + c];
        return;
    }
    const AemMaterial *m0 = P.mat + i0, *m1 = P.mat + i1, *m2 = P.mat + i2, *m3 = P.mat + i3;
    const float e = (m0->eps[c] + m1->eps[c] + m2->eps[c] + m3->eps[c]) / 4.0f;
    const float s = (m0->sig[c] + m1->sig[c] + m2->sig[c] + m3->sig[c]) / 4.0f;
    const float tp = 0.0f;
    ga = d_ga(s + tp, e, P.dt);
    gb = d_gb(s + tp, e, P.dt);
}

// E_new of one cell and one component (k_update_e's expressions)
__device__ __noinline__ float y4_e_comp(const AemParams& P, const float* gab, int comp, int px, int py, int pz, float eold,
                                        float d1, float d2, float den1, float den2, int i0, int i1, int i2, int i3) {
    const float curl = d1 * den1 + d2 * den2;
    float ga, gb;
    y4_gagb(P, gab, comp, i0, i1, i2, i3, ga, gb);
    float e = ga * eold + gb * curl;
    const int i = px + 1, j = py + 1, k = pz + 1;
    const int qxl = (i >= 2 && i <= P.npml[0][0]) ? i : 0, qxh = (i >= P.X + 1 - P.npml[0][1] && i <= P.X - 1) ? P.X + 1 - i : 0;
    const int qyl = (j >= 2 && j <= P.npml[1][0]) ? j : 0, qyh = (j >= P.Y + 1 - P.npml[1][1] && j <= P.Y - 1) ? P.Y + 1 - j : 0;
    const int qzl = (k >= 2 && k <= P.npml[2][0]) ? k : 0, qzh = (k >= P.Z + 1 - P.npml[2][1] && k <= P.Z - 1) ? P.Z + 1 - k : 0;
    // slab axes: Ex (y then z), Ey (x then z), Ez (x then y)
    const int a1 = comp == 0 ? 1 : 0, a2 = comp == 2 ? 1 : 2;
    const int q1l = a1 == 0 ? qxl : qyl, q1h = a1 == 0 ? qxh : qyh;
    const int q2l = a2 == 1 ? qyl : qzl, q2h = a2 == 1 ? qyh : qzh;
    if (q1l) e = e + gb * psi4(P.psi_e[comp][a1][0], P.psi_e[comp][a1][0], true, P.be[a1][0][q1l - 1], P.ce[a1][0][q1l - 1], d1, P.del[a1], psi_idx(P, a1, q1l, px, py, pz, P.npml[a1][0]));
    if (q1h) e = e + gb * psi4(P.psi_e[comp][a1][1], P.psi_e[comp][a1][1], true, P.be[a1][1][q1h - 1], P.ce[a1][1][q1h - 1], d1, P.del[a1], psi_idx(P, a1, q1h, px, py, pz, P.npml[a1][1]));
    if (q2l) e = e + gb * psi4(P.psi_e[comp][a2][0], P.psi_e[comp][a2][0], true, P.be[a2][0][q2l - 1], P.ce[a2][0][q2l - 1], d2, P.del[a2], psi_idx(P, a2, q2l, px, py, pz, P.npml[a2][0]));
    if (q2h) e = e + gb * psi4(P.psi_e[comp][a2][1], P.psi_e[comp][a2][1], true, P.be[a2][1][q2h - 1], P.ce[a2][1][q2h - 1], d2, P.del[a2], psi_idx(P, a2, q2h, px, py, pz, P.npml[a2][1]));
    return e;
}

// the -x halo cell (x0-1, py) of a row: Hy, Hz (never stored); dhx is
// den_h x of x0-1.  A bulk cell is computed here from the tiles; a CPML cell
// takes the per-cell path.
__device__ __forceinline__ float2 y4_h_xhalo(const AemParams& P, const float* E0, const float* E1, const float* Ho, int r,
                                             int x0, int py, int pz, int hzm, bool cpml_yz, float dhx, float dhy,
                                             float dhz) {
    const int c3 = 3;  // tile column of x0-1
    const float hyv = Ho[1 * Y4_HC + r * Y4_HW + c3];
    const float hzv = Ho[2 * Y4_HC + r * Y4_HW + c3];
    const int px = x0 - 1, i = x0;
    if (px < 0 || px > P.SX - 2 || py < 0 || py > P.SY - 2 || pz > hzm) return make_float2(hyv, hzv);
    const float* Ex = E0 + 0 * Y4_EC + r * Y4_EW;
    const float* Ey = E0 + 1 * Y4_EC + r * Y4_EW;
    const float* Ez = E0 + 2 * Y4_EC + r * Y4_EW;
    const float ex = Ex[c3], ey = Ey[c3], ez = Ez[c3];
    const float ex_jp = Ex[Y4_EW + c3], ey_ip = Ey[c3 + 1], ez_ip = Ez[c3 + 1];
    const float ex_kp = E1[0 * Y4_EC + r * Y4_EW + c3];
    if (!cpml_yz && i > P.npml[0][0] - 1 && i < P.X + 1 - P.npml[0][1]) {
        const float DB = P.DB;
        return make_float2(hyv + DB * ((ez_ip - ez) * dhx + (ex - ex_kp) * dhz),
                           hzv + DB * ((ey - ey_ip) * dhx + (ex_jp - ex) * dhy));
    }
    const float3 h = y4_h_cell(P, px, py, pz, ex, ey, ez, ex_jp, Ez[Y4_EW + c3], ey_ip, ez_ip, ex_kp,
                               E1[1 * Y4_EC + r * Y4_EW + c3], Ho[0 * Y4_HC + r * Y4_HW + c3], hyv, hzv, false);
    return make_float2(h.y, h.z);
}

// per-thread constants of the z march
struct Y4Row {
    int r, py, xb, xi, xbi;
    bool own;        // an owned-row warp on a stored row
    bool hrow;       // the row computes H (own rows and the -y halo row)
    unsigned hmask;  // cells of the group inside the H update range in x and y (bit e: cell xb+e)
    bool h_xpml;     // a cell of the group lies in an x CPML slab (H)
    int qyh_lo, qyh_hi;  // y CPML depth of the row (H), 0 outside
    unsigned emx, emy, emz;  // cells whose Ex / Ey / Ez is updated, as far as x and y decide
    bool unavg_xy;   // a cell of the group has i == 1 or j == 1 (no material averaging)
    bool e_xpml;     // a cell of the group lies in an x CPML slab (E)
    int qye_lo, qye_hi;  // y CPML depth of the row (E)
    long long rowoff;    // py * PX + xb
};

// H_new of the thread's four cells (row r of the tile) from E0 (plane k),
// E1 (k+1), Ho (H_old k); non-updated cells keep H_old.  `store`: write to
// H2 / psi_h2 (owned cells).  IN: the tile and plane lie inside the update
// range and outside every CPML slab (no masks, no CPML terms).
template <bool IN>
__device__ __forceinline__ void y4_h_group(const AemParams& P, const Y4Row& T, const float* E0, const float* E1,
                                           const float* Ho, int pz, int hzm, float dhz, const float* dxs, float dhy,
                                           bool store, float hx[4], float hy[4], float hz[4]) {
    const float* Ex = E0 + 0 * Y4_EC + T.r * Y4_EW;
    const float* Ey = E0 + 1 * Y4_EC + T.r * Y4_EW;
    const float* Ez = E0 + 2 * Y4_EC + T.r * Y4_EW;
    const float4 ex = lds4(Ex + T.xi), ey = lds4(Ey + T.xi), ez = lds4(Ez + T.xi);
    const float4 exj = lds4(Ex + Y4_EW + T.xi), ezj = lds4(Ez + Y4_EW + T.xi);
    const float ey4 = Ey[T.xi + 4], ez4 = Ez[T.xi + 4];
    const float4 exk = lds4(E1 + 0 * Y4_EC + T.r * Y4_EW + T.xi), eyk = lds4(E1 + 1 * Y4_EC + T.r * Y4_EW + T.xi);
    const float4 h0x = lds4(Ho + 0 * Y4_HC + T.r * Y4_HW + T.xi), h0y = lds4(Ho + 1 * Y4_HC + T.r * Y4_HW + T.xi),
                 h0z = lds4(Ho + 2 * Y4_HC + T.r * Y4_HW + T.xi);
    const float vex[4] = {ex.x, ex.y, ex.z, ex.w}, vey[4] = {ey.x, ey.y, ey.z, ey.w}, vez[4] = {ez.x, ez.y, ez.z, ez.w};
    const float vexj[4] = {exj.x, exj.y, exj.z, exj.w}, vezj[4] = {ezj.x, ezj.y, ezj.z, ezj.w};
    const float veyi[4] = {ey.y, ey.z, ey.w, ey4}, vezi[4] = {ez.y, ez.z, ez.w, ez4};
    const float vexk[4] = {exk.x, exk.y, exk.z, exk.w}, veyk[4] = {eyk.x, eyk.y, eyk.z, eyk.w};
    const float vhx[4] = {h0x.x, h0x.y, h0x.z, h0x.w}, vhy[4] = {h0y.x, h0y.y, h0y.z, h0y.w},
                vhz[4] = {h0z.x, h0z.y, h0z.z, h0z.w};
    // cells of the group inside the H update range (all four in the bulk)
    const unsigned mk = IN ? 0xFu : (pz <= hzm ? T.hmask : 0u);
    if (!IN && !mk) {
#pragma unroll
        for (int e = 0; e < 4; e++) { hx[e] = vhx[e]; hy[e] = vhy[e]; hz[e] = vhz[e]; }
        return;
    }
    const float DB = P.DB;
    const float4 dx4 = lds4(dxs + 4 * (T.xi / 4 - 1));
    const float dhx[4] = {dx4.x, dx4.y, dx4.z, dx4.w};
#pragma unroll
    for (int e = 0; e < 4; e++) {
        hx[e] = vhx[e] + DB * ((vez[e] - vezj[e]) * dhy + (veyk[e] - vey[e]) * dhz);
        hy[e] = vhy[e] + DB * ((vezi[e] - vez[e]) * dhx[e] + (vex[e] - vexk[e]) * dhz);
        hz[e] = vhz[e] + DB * ((vey[e] - veyi[e]) * dhx[e] + (vexj[e] - vex[e]) * dhy);
    }
    if constexpr (IN) {
        if (store) {
            const long long c = (long long)pz * P.plane + T.rowoff;
            *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.H2[0]) + c) = make_float4(hx[0], hx[1], hx[2], hx[3]);
            *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.H2[1]) + c) = make_float4(hy[0], hy[1], hy[2], hy[3]);
            *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.H2[2]) + c) = make_float4(hz[0], hz[1], hz[2], hz[3]);
        }
        return;
    }
    // CPML terms in the reference's order: Hx (y, z), Hy (x, z), Hz (x, y)
    if (T.h_xpml) {
        float dzx[4], dyx[4];
#pragma unroll
        for (int e = 0; e < 4; e++) { dzx[e] = vezi[e] - vez[e]; dyx[e] = vey[e] - veyi[e]; }
        y4_h_xpml4(P, T.xb, T.py, pz, mk, dzx, dyx, store, hy, hz);
    }
    if (T.qyh_lo | T.qyh_hi) {
        float dzy[4], dxy[4];
#pragma unroll
        for (int e = 0; e < 4; e++) { dzy[e] = vez[e] - vezj[e]; dxy[e] = vexj[e] - vex[e]; }
        for (int s = 0; s < 2; s++) {
            const int q = s ? T.qyh_hi : T.qyh_lo;
            if (!q) continue;
            const int n = P.npml[1][s];
            const long long o = ((long long)pz * n + (q - 1)) * P.PX + T.xb;
            y4_psi_row2(P.psi_h[0][1][s], P.psi_h2[0][1][s], mk, dzy, DB, hx, P.psi_h[2][1][s], P.psi_h2[2][1][s], mk, dxy,
                        DB, hz, store, P.bh[1][s][q - 1], P.ch[1][s][q - 1], P.del[1], o);
        }
    }
    const int k = pz + 1;
    const int qz_lo = (k <= P.npml[2][0] - 1) ? k : 0, qz_hi = (k >= P.Z + 1 - P.npml[2][1]) ? P.Z - k : 0;
    if (qz_lo | qz_hi) {
        float dyz[4], dxz[4];
#pragma unroll
        for (int e = 0; e < 4; e++) { dyz[e] = veyk[e] - vey[e]; dxz[e] = vex[e] - vexk[e]; }
        for (int s = 0; s < 2; s++) {
            const int q = s ? qz_hi : qz_lo;
            if (!q) continue;
            const long long o = ((long long)(q - 1) * P.SY + T.py) * P.PX + T.xb;
            y4_psi_row2(P.psi_h[0][2][s], P.psi_h2[0][2][s], mk, dyz, DB, hx, P.psi_h[1][2][s], P.psi_h2[1][2][s], mk, dxz,
                        DB, hy, store, P.bh[2][s][q - 1], P.ch[2][s][q - 1], P.del[2], o);
        }
    }
    if (mk != 0xFu) {
#pragma unroll
        for (int e = 0; e < 4; e++)
            if (!(mk >> e & 1u)) { hx[e] = vhx[e]; hy[e] = vhy[e]; hz[e] = vhz[e]; }
    }
    if (store) {
        const long long c = (long long)pz * P.plane + T.rowoff;
        y4_store4(P.H2[0], c, mk, hx);
        y4_store4(P.H2[1], c, mk, hy);
        y4_store4(P.H2[2], c, mk, hz);
    }
}

__global__ void __launch_bounds__(Y4_NT, 1) k_yee4(const __grid_constant__ AemParams P, const __grid_constant__ Y4Maps M) {
    extern __shared__ __align__(128) unsigned char smem[];
    float* Hn = reinterpret_cast<float*>(smem + Y4_OFF_HN);    // [2][16][128]: hx, hz of H_new(k)
    float* dzs = reinterpret_cast<float*>(smem + Y4_OFF_DZ);   // den_h z, den_e z of the chunk's planes
    float* dxs = reinterpret_cast<float*>(smem + Y4_OFF_DX);   // den_h x, den_e x of the tile's columns
    float* xh = reinterpret_cast<float*>(smem + Y4_OFF_XH);    // [plane & 1][row 1..15][Hy, Hz] of the -x halo cell
    float* gab = reinterpret_cast<float*>(smem + Y4_OFF_GAB);  // [mat][6]: ga xyz, gb xyz
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + Y4_OFF_BAR);
    const int lane = threadIdx.x, w = threadIdx.y;
    const int tid = lane + 32 * w;
    const int x0 = blockIdx.x * Y4_TX, y0 = blockIdx.y * Y4_TY;
    const int z0 = blockIdx.z * Y4_ZC, z1 = min(P.SZ, z0 + Y4_ZC);
    const int hzm = P.per[2] ? P.SZ - 1 : P.SZ - 2;
    const unsigned FULL = 0xffffffffu;
    if (y4_sa(smem) & 127) {  // the TMA boxes need 128-byte aligned destinations
        if (tid == 0) atomicAdd(P.err, 1);
        return;
    }
    auto zw = [&](int p) { return P.per[2] ? (p % P.SZ + P.SZ) % P.SZ : p; };
    auto md = [](int p, int m) { return ((p % m) + m) % m; };
    auto Ew = [&](int p) { return reinterpret_cast<float*>(smem + md(p, Y4_ES) * 3 * Y4_EC * 4); };
    auto Hw = [&](int p) { return reinterpret_cast<float*>(smem + Y4_OFF_H + md(p, Y4_HS) * 3 * Y4_HC * 4); };
    auto Iw = [&](int p) { return smem + Y4_OFF_I + md(p, Y4_IS) * Y4_IC; };
    // E (3 boxes), H (3) and ids (1) of plane p into the given slots (null: skipped)
    auto issue = [&](float* E, float* H, unsigned char* I, int p, uint64_t* b) {
        for (int c = 0; c < 3; c++)
            if (E) y4_tma(E + c * Y4_EC, &M.e[c], x0 - 4, y0 - 1, p, b);
        for (int c = 0; c < 3; c++)
            if (H) y4_tma(H + c * Y4_HC, &M.h[c], x0 - 4, y0 - 1, p, b);
        if (I) y4_tma(I, &M.id, x0 - 16, y0 - 1, p, b);
    };
    const bool below = P.per[2] || z0 > 0;
    auto pz_of = [&](int p) { return (p < 0 || p >= P.SZ) && !P.per[2] ? -1 : zw(p); };  // -1: zero fill

    if (tid == 0) {
        for (int b = 0; b < Y4_NB; b++) y4_bar_init(&bar[b]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int q = tid; q < P.nmat * 6; q += Y4_NT) {
        const int m = q / 6, c = q % 6;
        gab[q] = c < 3 ? P.ucoef[m].ga[c] : P.ucoef[m].gb[c - 3];
    }
    for (int q = tid; q < z1 - z0; q += Y4_NT) {
        dzs[q] = P.den_h[2][zw(z0 + q)];
        dzs[Y4_ZC + q] = P.den_e[2][zw(z0 + q)];
    }
    for (int q = tid; q < Y4_TX; q += Y4_NT) {
        const bool in = x0 + q < P.SX;
        dxs[q] = in ? P.den_h[0][x0 + q] : 0.0f;
        dxs[Y4_TX + q] = in ? P.den_e[0][x0 + q] : 0.0f;
    }
    if (tid == 0) dxs[2 * Y4_TX] = x0 >= 1 ? P.den_h[0][x0 - 1] : 0.0f;
    __syncthreads();
    if (tid == 0) {
        y4_bar_expect(&bar[0], Y4_TX_FIRST);
        issue(Ew(z0 - 1), Hw(z0 - 1), Iw(z0 - 1), below ? zw(z0 - 1) : -1, &bar[0]);
        issue(Ew(z0), Hw(z0), Iw(z0), zw(z0), &bar[0]);
        issue(Ew(z0 + 1), nullptr, nullptr, pz_of(z0 + 1), &bar[0]);
        for (int t = z0 + 1; t < z0 + Y4_LA && t < z1; t++) {
            y4_bar_expect(&bar[t - z0], Y4_TX_STAGE);
            issue(Ew(t + 1), nullptr, nullptr, pz_of(t + 1), &bar[t - z0]);
            issue(nullptr, Hw(t), Iw(t), zw(t), &bar[t - z0]);
        }
    }

    // per-thread constants
    Y4Row T;
    T.r = w == Y4_TY ? 0 : w + 1;
    T.py = y0 - 1 + T.r;
    T.xb = x0 + 4 * lane;
    T.xi = 4 * lane + 4;
    T.xbi = 4 * lane + 16;
    T.own = w < Y4_TY && T.py < P.SY;
    T.hrow = T.own || (w == Y4_TY && T.py >= 0);
    T.rowoff = (long long)T.py * P.PX + T.xb;
    const int j = T.py + 1, i0 = T.xb + 1;
    {
        unsigned hx = 0, ex = 0, eyz = 0;
        for (int e = 0; e < 4; e++) {
            const int px = T.xb + e;
            if (px <= P.SX - 2) { hx |= 1u << e; ex |= 1u << e; }
            if (px >= 1 && px <= P.SX - 2) eyz |= 1u << e;
        }
        const bool rx = T.py >= 1 && T.py <= P.SY - 2, ry = T.py >= 0 && T.py <= P.SY - 2;
        T.hmask = ry ? hx : 0u;
        T.emx = rx ? ex : 0u;
        T.emy = ry ? eyz : 0u;
        T.emz = rx ? eyz : 0u;
        T.unavg_xy = T.xb == 0 || T.py == 0;
    }
    T.h_xpml = i0 <= P.npml[0][0] - 1 || i0 + 3 >= P.X + 1 - P.npml[0][1];
    T.qyh_lo = (j <= P.npml[1][0] - 1) ? j : 0;
    T.qyh_hi = (j >= P.Y + 1 - P.npml[1][1]) ? P.Y - j : 0;
    T.e_xpml = i0 <= P.npml[0][0] || i0 + 3 >= P.X + 1 - P.npml[0][1];
    T.qye_lo = (j >= 2 && j <= P.npml[1][0]) ? j : 0;
    T.qye_hi = (j >= P.Y + 1 - P.npml[1][1] && j <= P.Y - 1) ? P.Y + 1 - j : 0;
    const bool yin = T.py >= 0 && T.py < P.SY;
    const float dhy = yin ? P.den_h[1][T.py] : 0.0f, dey = yin ? P.den_e[1][T.py] : 0.0f;
    // the tile (with its -x / -y halo) inside the update range and outside
    // the x and y CPML slabs of H and E (reference indices x0..x0+128,
    // y0..y0+15)
    const bool tile_in = x0 >= 1 && x0 + Y4_TX - 1 <= P.SX - 2 && x0 > P.npml[0][0] &&
                         x0 + Y4_TX < P.X + 1 - P.npml[0][1] && y0 >= 1 && y0 + Y4_TY - 1 <= P.SY - 2 &&
                         y0 > P.npml[1][0] && y0 + Y4_TY < P.Y + 1 - P.npml[1][1];
    // H_new(k) (Hy, Hz) of the -x halo cells of rows y0..y0+14, one per
    // lane 0..14 of the halo warp, into xh[k & 1]; that warp has no E update,
    // so this runs while the others update E of the plane before
    auto xhalo_rows = [&](int k) {
        if (lane >= Y4_TY) return;
        const int py = y0 + lane;
        float hyv = 0.0f, hzv = 0.0f;
        if (py < P.SY) {
            const int pz = zw(k), kz = pz + 1, jr = py + 1;
            const bool cpml_yz = jr <= P.npml[1][0] - 1 || jr >= P.Y + 1 - P.npml[1][1] || kz <= P.npml[2][0] - 1 ||
                                 kz >= P.Z + 1 - P.npml[2][1];
            const float2 hh = y4_h_xhalo(P, Ew(k), Ew(k + 1), Hw(k), lane + 1, x0, py, pz, hzm, cpml_yz, dxs[2 * Y4_TX],
                                         P.den_h[1][py], dzs[k - z0]);
            hyv = hh.x; hzv = hh.y;
        }
        xh[((k & 1) * Y4_TY + lane) * 2 + 0] = hyv;
        xh[((k & 1) * Y4_TY + lane) * 2 + 1] = hzv;
    };

    bool ok = y4_bar_wait(&bar[0], 0);
    if (!__syncthreads_and(ok)) {
        if (tid == 0) atomicAdd(P.err, 1);
        return;
    }
    // H_new(z0-1) of the own cells (the plane below belongs to the chunk underneath)
    float hxp[4] = {0, 0, 0, 0}, hyp[4] = {0, 0, 0, 0};
    if (below && T.own) {
        float hz_unused[4];
        const int pzb = zw(z0 - 1);
        y4_h_group<false>(P, T, Ew(z0 - 1), Ew(z0), Hw(z0 - 1), pzb, hzm, P.den_h[2][pzb], dxs, dhy, false, hxp, hyp, hz_unused);
    }
    if (w == Y4_TY) xhalo_rows(z0);

    for (int k = z0; k < z1; k++) {
        const int pz = zw(k);
        // stage k (E(k+1), H(k), ids(k)) has landed, and every thread is done
        // with plane k-1: stage k+Y4_LA reuses the slots of E(k-1), H(k-1),
        // ids(k-2) and the barrier of stage k-1
        if (k > z0) ok = y4_bar_wait(&bar[(k - z0) % Y4_NB], ((k - z0) / Y4_NB) & 1);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) atomicAdd(P.err, 1);
            return;
        }
        if (tid == 0 && k + Y4_LA < z1) {
            const int t = k + Y4_LA;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            uint64_t* b = &bar[(t - z0) % Y4_NB];
            y4_bar_expect(b, Y4_TX_STAGE);
            issue(Ew(t + 1), nullptr, nullptr, pz_of(t + 1), b);
            issue(nullptr, Hw(t), Iw(t), zw(t), b);
        }

        // the plane's update: IN (tile and plane inside the update range and
        // outside every CPML slab) drops the masks and CPML terms
        float hx[4], hy[4], hz[4];
        auto plane = [&](auto in_tag) {
            constexpr bool IN = decltype(in_tag)::value;
            // ---- H_new(k): own rows and the -y halo row (halo warp)
            const float* E0 = Ew(k);
            const float dhz = dzs[k - z0], dez = dzs[Y4_ZC + k - z0];
            if (T.hrow)
                y4_h_group<IN>(P, T, E0, Ew(k + 1), Hw(k), pz, hzm, dhz, dxs, dhy, T.own, hx, hy, hz);
            else
                for (int e = 0; e < 4; e++) hx[e] = hy[e] = hz[e] = 0.0f;
            *reinterpret_cast<float4*>(Hn + (0 * Y4_HR + T.r) * Y4_TX + 4 * lane) = make_float4(hx[0], hx[1], hx[2], hx[3]);
            *reinterpret_cast<float4*>(Hn + (1 * Y4_HR + T.r) * Y4_TX + 4 * lane) = make_float4(hz[0], hz[1], hz[2], hz[3]);
            __syncthreads();

            // ---- E_new(k) of the own rows; the halo warp meanwhile computes the -x
            // halo cells of plane k+1
            if (w == Y4_TY && k + 1 < z1) {
                // stage k+1 (E(k+2), H(k+1)) may not have landed yet
                ok = y4_bar_wait(&bar[(k + 1 - z0) % Y4_NB], ((k + 1 - z0) / Y4_NB) & 1) && ok;
                if (ok) xhalo_rows(k + 1);
            }
            if (w < Y4_TY) {
                float hz_im0 = __shfl_up_sync(FULL, hz[3], 1), hy_im0 = __shfl_up_sync(FULL, hy[3], 1);
                if (lane == 0) {
                    hy_im0 = xh[((k & 1) * Y4_TY + w) * 2 + 0];
                    hz_im0 = xh[((k & 1) * Y4_TY + w) * 2 + 1];
                }
                if (T.own) {
                    const int r = T.r;
                    const float4 hxj4 = lds4(Hn + (0 * Y4_HR + r - 1) * Y4_TX + 4 * lane);
                    const float4 hzj4 = lds4(Hn + (1 * Y4_HR + r - 1) * Y4_TX + 4 * lane);
                    const float hxj[4] = {hxj4.x, hxj4.y, hxj4.z, hxj4.w}, hzj[4] = {hzj4.x, hzj4.y, hzj4.z, hzj4.w};
                    const float him_z[4] = {hz_im0, hz[0], hz[1], hz[2]}, him_y[4] = {hy_im0, hy[0], hy[1], hy[2]};
                    const float4 ex4 = lds4(E0 + 0 * Y4_EC + r * Y4_EW + T.xi), ey4 = lds4(E0 + 1 * Y4_EC + r * Y4_EW + T.xi),
                                 ez4 = lds4(E0 + 2 * Y4_EC + r * Y4_EW + T.xi);
                    const float vex[4] = {ex4.x, ex4.y, ex4.z, ex4.w}, vey[4] = {ey4.x, ey4.y, ey4.z, ey4.w},
                                vez[4] = {ez4.x, ez4.y, ez4.z, ez4.w};
                    const float4 dx4 = lds4(dxs + Y4_TX + 4 * lane);
                    const float dex[4] = {dx4.x, dx4.y, dx4.z, dx4.w};
                    const unsigned char* I0 = Iw(k);
                    const unsigned char* I1 = Iw(k - 1);
                    const unsigned char* a0 = I0 + r * Y4_IW + T.xbi;        // plane k, row r
                    const unsigned char* a1 = I0 + (r - 1) * Y4_IW + T.xbi;  // plane k, row r-1
                    const unsigned char* b0 = I1 + r * Y4_IW + T.xbi;        // plane k-1, row r
                    const unsigned char* b1 = I1 + (r - 1) * Y4_IW + T.xbi;  // plane k-1, row r-1
                    const unsigned w_a0 = *reinterpret_cast<const unsigned*>(a0), w_a1 = *reinterpret_cast<const unsigned*>(a1);
                    const unsigned w_b0 = *reinterpret_cast<const unsigned*>(b0), w_b1 = *reinterpret_cast<const unsigned*>(b1);
                    const int kk = pz + 1;
                    // cells whose Ex / Ey / Ez this step updates
                    const bool zxy = P.per[2] || (pz >= 1 && pz <= P.SZ - 2), zz = P.per[2] || pz <= P.SZ - 2;
                    const unsigned mx = IN ? 0xFu : zxy ? T.emx : 0u, my = IN ? 0xFu : zxy ? T.emy : 0u,
                                   mz = IN ? 0xFu : zz ? T.emz : 0u;
                    const unsigned m = w_a0 & 0xffu;
                    const unsigned rep = m * 0x01010101u;
                    // one material around every cell; a cell on an index-1 plane
                    // uses material 0 without averaging, so there the group's
                    // material must be 0
                    const bool uniform = w_a0 == rep && w_a1 == rep && w_b0 == rep && w_b1 == rep && a0[-1] == m &&
                                         a1[-1] == m && b0[-1] == m &&
                                         (IN || m == 0 || !(T.unavg_xy || (!P.per[2] && kk == 1)));
                    if (!IN && !(mx | my | mz)) {
                    } else if (uniform) {
                        const float gax = gab[m * 6 + 0], gay = gab[m * 6 + 1], gaz = gab[m * 6 + 2];
                        const float gbx = gab[m * 6 + 3], gby = gab[m * 6 + 4], gbz = gab[m * 6 + 5];
                        float ex_n[4], ey_n[4], ez_n[4];
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            ex_n[e] = gax * vex[e] + gbx * ((hz[e] - hzj[e]) * dey + (hyp[e] - hy[e]) * dez);
                            ey_n[e] = gay * vey[e] + gby * ((him_z[e] - hz[e]) * dex[e] + (hx[e] - hxp[e]) * dez);
                            ez_n[e] = gaz * vez[e] + gbz * ((hy[e] - him_y[e]) * dex[e] + (hxj[e] - hx[e]) * dey);
                        }
                        if constexpr (IN) {
                            const long long c = (long long)pz * P.plane + T.rowoff;
                            *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.E2[0]) + c) = make_float4(ex_n[0], ex_n[1], ex_n[2], ex_n[3]);
                            *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.E2[1]) + c) = make_float4(ey_n[0], ey_n[1], ey_n[2], ey_n[3]);
                            *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.E2[2]) + c) = make_float4(ez_n[0], ez_n[1], ez_n[2], ez_n[3]);
                            return;
                        }
                        // CPML terms in the reference's order: Ex (y, z), Ey (x, z), Ez (x, y)
                        if (T.e_xpml) {
                            float dzx[4], dyx[4];
#pragma unroll
                            for (int e = 0; e < 4; e++) { dzx[e] = him_z[e] - hz[e]; dyx[e] = hy[e] - him_y[e]; }
                            y4_e_xpml4(P, T.xb, T.py, pz, my, mz, dzx, dyx, gby, gbz, ey_n, ez_n);
                        }
                        if (T.qye_lo | T.qye_hi) {
                            float dzy[4], dxy[4];
#pragma unroll
                            for (int e = 0; e < 4; e++) { dzy[e] = hz[e] - hzj[e]; dxy[e] = hxj[e] - hx[e]; }
                            for (int s = 0; s < 2; s++) {
                                const int q = s ? T.qye_hi : T.qye_lo;
                                if (!q) continue;
                                const int n = P.npml[1][s];
                                const long long o = ((long long)pz * n + (q - 1)) * P.PX + T.xb;
                                y4_psi_row2(P.psi_e[0][1][s], P.psi_e[0][1][s], mx, dzy, gbx, ex_n, P.psi_e[2][1][s], P.psi_e[2][1][s], mz,
                                            dxy, gbz, ez_n, true, P.be[1][s][q - 1], P.ce[1][s][q - 1], P.del[1], o);
                            }
                        }
                        const int qzl = (kk >= 2 && kk <= P.npml[2][0]) ? kk : 0;
                        const int qzh = (kk >= P.Z + 1 - P.npml[2][1] && kk <= P.Z - 1) ? P.Z + 1 - kk : 0;
                        if (qzl | qzh) {
                            float dyz[4], dxz[4];
#pragma unroll
                            for (int e = 0; e < 4; e++) { dyz[e] = hyp[e] - hy[e]; dxz[e] = hx[e] - hxp[e]; }
                            for (int s = 0; s < 2; s++) {
                                const int q = s ? qzh : qzl;
                                if (!q) continue;
                                const long long o = ((long long)(q - 1) * P.SY + T.py) * P.PX + T.xb;
                                y4_psi_row2(P.psi_e[0][2][s], P.psi_e[0][2][s], mx, dyz, gbx, ex_n, P.psi_e[1][2][s], P.psi_e[1][2][s], my,
                                            dxz, gby, ey_n, true, P.be[2][s][q - 1], P.ce[2][s][q - 1], P.del[2], o);
                            }
                        }
                        const long long c = (long long)pz * P.plane + T.rowoff;
                        if (mx) y4_store4(P.E2[0], c, mx, ex_n);
                        if (my) y4_store4(P.E2[1], c, my, ey_n);
                        if (mz) y4_store4(P.E2[2], c, mz, ez_n);
                    } else {
                        const int py = T.py;
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            const int px = T.xb + e, i = px + 1;
                            if (px >= P.SX) continue;
                            const bool ex_u = px <= P.SX - 2 && py >= 1 && py <= P.SY - 2 && (P.per[2] || (pz >= 1 && pz <= P.SZ - 2));
                            const bool ey_u = px >= 1 && px <= P.SX - 2 && py <= P.SY - 2 && (P.per[2] || (pz >= 1 && pz <= P.SZ - 2));
                            const bool ez_u = px >= 1 && px <= P.SX - 2 && py >= 1 && py <= P.SY - 2 && (P.per[2] || pz <= P.SZ - 2);
                            if (!(ex_u || ey_u || ez_u)) continue;
                            const bool unavg = i == 1 || j == 1 || (!P.per[2] && kk == 1);
                            const int idc = unavg ? 0 : a0[e], idx_ = unavg ? 0 : a0[e - 1], idy_ = unavg ? 0 : a1[e],
                                      idxy = unavg ? 0 : a1[e - 1];
                            const int pdc = unavg ? 0 : b0[e], pdx = unavg ? 0 : b0[e - 1], pdy = unavg ? 0 : b1[e];
                            const long long c = lin(P, px, py, pz);
                            if (ex_u) stf4(P.E2[0], c, y4_e_comp(P, gab, 0, px, py, pz, vex[e], hz[e] - hzj[e], hyp[e] - hy[e], dey, dez, idc, idy_, pdc, pdy));
                            if (ey_u) stf4(P.E2[1], c, y4_e_comp(P, gab, 1, px, py, pz, vey[e], him_z[e] - hz[e], hx[e] - hxp[e], dex[e], dez, idc, idx_, pdc, pdx));
                            if (ez_u) stf4(P.E2[2], c, y4_e_comp(P, gab, 2, px, py, pz, vez[e], hy[e] - him_y[e], hxj[e] - hx[e], dex[e], dey, idc, idx_, idy_, idxy));
                        }
                    }
                }
            }
        };
        const int kz = pz + 1;
        const bool plane_in = (P.per[2] || (pz >= 1 && pz <= P.SZ - 2)) && pz <= hzm && kz > P.npml[2][0] &&
                              kz < P.Z + 1 - P.npml[2][1];
        if (tile_in && plane_in)
            plane(std::true_type{});
        else
            plane(std::false_type{});
#pragma unroll
        for (int e = 0; e < 4; e++) { hxp[e] = hx[e]; hyp[e] = hy[e]; }
    }
}

// ---- host side ----

static PFN_cuTensorMapEncodeTiled_v12000 y4_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// 3-D map over a [SZ][SY][PX] array of `esize`-byte elements, box bx x by x 1
static void y4_map(CUtensorMap* m, const void* base, CUtensorMapDataType t, int esize, const AemParams& P, int bx, int by) {
    auto enc = y4_encoder();
    if (!enc) throw std::runtime_error("cuTensorMapEncodeTiled is not available from the CUDA driver");
    const cuuint64_t dims[3] = {(cuuint64_t)P.PX, (cuuint64_t)P.SY, (cuuint64_t)P.SZ};
    const cuuint64_t strides[2] = {(cuuint64_t)P.PX * esize, (cuuint64_t)P.PX * P.SY * esize};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(m, t, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

int launch_yee4(const AemParams& P, cudaStream_t s) {
    static bool attr_set[64] = {};
    static std::mutex mu;
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> g(mu);
        if (dev >= 0 && dev < 64 && !attr_set[dev]) {
            cudaFuncSetAttribute(k_yee4, cudaFuncAttributeMaxDynamicSharedMemorySize, Y4_SMEM);
            cudaFuncSetAttribute(k_yee4, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
            attr_set[dev] = true;
        }
    }
    if (!P.err) throw std::runtime_error("fused kernel launched without an error counter");
    Y4Maps M;
    for (int c = 0; c < 3; c++) {
        y4_map(&M.e[c], P.E[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, P, Y4_EW, Y4_ER);
        y4_map(&M.h[c], P.H[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, P, Y4_HW, Y4_HR);
    }
    y4_map(&M.id, P.cell, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, P, Y4_IW, Y4_IR);
    // the last position of a non-periodic axis is never updated: no tile for it
    const int ux = P.SX - 1, uy = P.SY - 1, uz = P.per[2] ? P.SZ : P.SZ - 1;
    dim3 blk(32, Y4_TY + 1), grd((ux + Y4_TX - 1) / Y4_TX, (uy + Y4_TY - 1) / Y4_TY, (uz + Y4_ZC - 1) / Y4_ZC);
    k_yee4<<<grd, blk, Y4_SMEM, s>>>(P, M);
    return 1;
}

}  // namespace aem
