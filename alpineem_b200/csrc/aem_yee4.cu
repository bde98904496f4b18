// aem_yee4.cu -- fused H+E step, 4 cells per thread (grids without x/y
// periodicity; any z).
//
// Same arithmetic, statement for statement, as k_update_h / k_update_e
// (bulk curl fdtd_solver.f90:4442-4484 / :5667-5710, CPML :5227-5375 /
// :6522-6670), so the fields are bit-identical to the other paths.
//
// A CTA owns a 128 x 8 (x, y) column tile and marches a z chunk.  Warps 0..7
// own rows y0..y0+7; lane l owns the four cells x0+4l .. x0+4l+3, so every
// shared-memory and global access of a cell group is one 16-byte operation.
// Warp 8 computes the -y halo row of H (y0-1), which the E update of row y0
// needs; lane 0 of warps 0..7 computes the -x halo cell (x0-1).  Per plane
// p, a ring slot receives by cp.async (16-byte chunks, zero-filled off the
// grid): E_old(p) on rows y0-1..y0+8, x0-4..x0+131; H_old(p) on rows
// y0-1..y0+7, x0-4..x0+127; the material ids of rows y0-1..y0+7,
// x0-16..x0+127.  Plane k+2 is requested while plane k is computed.  Fields
// and H-psi are double-buffered (read E/H/psi_h, write E2/H2/psi_h2), so halo
// values recomputed here never race with their owners' stores.
//
// Per cell group the fast path covers interior cells outside the CPML whose
// seven surrounding cells share one material (ga/gb from a shared-memory
// copy of the material table); every other cell takes the per-cell path
// with the reference's 4-cell material average and the CPML terms.
#include <cstdlib>
#include <cstring>

#include "aem_dev.cuh"
#include "aem_kernels.h"

namespace aem {

constexpr int Y4_TX = 128, Y4_TY = 8, Y4_ZC = 64;
constexpr int Y4_EW = Y4_TX + 8, Y4_ER = Y4_TY + 2;  // E tile 136 x 10, x from x0-4
constexpr int Y4_HW = Y4_TX + 4, Y4_HR = Y4_TY + 1;  // H tile 132 x 9, x from x0-4
constexpr int Y4_IW = Y4_TX + 16;                    // ids 144 bytes x 9 rows, x from x0-16
// three rings: E planes k, k+1, k+2; H planes k, k+1; id planes k-1, k, k+1
constexpr int Y4_ES = 3, Y4_HS = 2, Y4_IS = 3;
constexpr int Y4_E_B = 3 * Y4_ER * Y4_EW * 4, Y4_H_B = 3 * Y4_HR * Y4_HW * 4, Y4_I_B = Y4_HR * Y4_IW;
constexpr int Y4_HN_F = 2 * Y4_HR * Y4_TX;  // H_new hx, hz of rows y0-1..y0+7
constexpr int Y4_NMAT = AEM_MAX_MATERIALS;
constexpr size_t Y4_OFF_H = (size_t)Y4_ES * Y4_E_B, Y4_OFF_I = Y4_OFF_H + (size_t)Y4_HS * Y4_H_B;
constexpr size_t Y4_OFF_HN = Y4_OFF_I + (size_t)Y4_IS * Y4_I_B;
constexpr size_t Y4_SMEM = Y4_OFF_HN + (size_t)Y4_HN_F * 4 + (size_t)Y4_NMAT * 6 * 4;
static_assert(Y4_E_B % 16 == 0 && Y4_H_B % 16 == 0 && Y4_I_B % 16 == 0, "tiles must stay 16-byte aligned");

__device__ inline float ldf4(const void* b, long long i) { return reinterpret_cast<const float*>(b)[i]; }
__device__ inline void stf4(void* b, long long i, float v) { reinterpret_cast<float*>(b)[i] = v; }
__device__ inline float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }

__device__ inline void cp16b(void* smem, const void* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ inline void cp_commit4() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ inline void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ inline float psi4(const void* rd, void* wr, bool store, float b, float c, float diff, float dl, long long q) {
    const float nw = b * ldf4(rd, q) + c * diff / dl;
    if (store) stf4(wr, q, nw);
    return nw;
}

// request the tiles of plane p (wrapped; -1 / SZ = absent): E into `E`,
// H into `H`, ids into `I` (a null destination skips that tile)
__device__ inline void y4_issue(const AemParams& P, float* E, float* H, unsigned char* I, int p, int x0, int y0) {
    const bool pv = p >= 0 && p < P.SZ;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x, nt = blockDim.x * blockDim.y;
    const int nE = E ? 3 * Y4_ER * (Y4_EW / 4) : 0, nH = H ? 3 * Y4_HR * (Y4_HW / 4) : 0, nI = I ? Y4_HR * (Y4_IW / 16) : 0;
    const long long pbase = pv ? (long long)p * P.plane : 0;
    for (int q = tid; q < nE + nH + nI; q += nt) {
        if (q < nE) {
            const int c = q / (Y4_ER * (Y4_EW / 4)), r = (q / (Y4_EW / 4)) % Y4_ER, ch = q % (Y4_EW / 4);
            const int x = x0 - 4 + 4 * ch, y = y0 - 1 + r;
            const bool ok = pv && x >= 0 && x + 4 <= P.PX && y >= 0 && y < P.SY;
            const float* src = reinterpret_cast<const float*>(P.E[c]) + (ok ? pbase + (long long)y * P.PX + x : 0);
            cp16b(E + (c * Y4_ER + r) * Y4_EW + 4 * ch, src, ok);
        } else if (q < nE + nH) {
            const int t = q - nE;
            const int c = t / (Y4_HR * (Y4_HW / 4)), r = (t / (Y4_HW / 4)) % Y4_HR, ch = t % (Y4_HW / 4);
            const int x = x0 - 4 + 4 * ch, y = y0 - 1 + r;
            const bool ok = pv && x >= 0 && x + 4 <= P.PX && y >= 0 && y < P.SY;
            const float* src = reinterpret_cast<const float*>(P.H[c]) + (ok ? pbase + (long long)y * P.PX + x : 0);
            cp16b(H + (c * Y4_HR + r) * Y4_HW + 4 * ch, src, ok);
        } else {
            const int t = q - nE - nH;
            const int r = t / (Y4_IW / 16), ch = t % (Y4_IW / 16);
            const int x = x0 - 16 + 16 * ch, y = y0 - 1 + r;
            const bool ok = pv && x >= 0 && x + 16 <= P.PX && y >= 0 && y < P.SY;
            const unsigned char* src = P.cell + (ok ? pbase + (long long)y * P.PX + x : 0);
            cp16b(I + r * Y4_IW + 16 * ch, src, ok);
        }
    }
}

// H_new of one cell (k_update_h's expressions; psi from psi_h, to psi_h2 when store)
__device__ __noinline__ float3 y4_h_cell(const AemParams& P, int px, int py, int pz, float ex, float ey, float ez,
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

// Ga/Gb of an E edge from its four cell ids (reference order, ref :2516-2527)
// CPML terms of one H cell added to bulk values (the k_update_h order:
// Hx y then z, Hy x then z, Hz x then y)
__device__ __noinline__ float3 y4_h_pml(const AemParams& P, int px, int py, int pz, float dzy, float dyz, float dzx,
                                        float dxz, float dyx, float dxy, bool store, float hxv, float hyv, float hzv) {
    // dzy = ez - ez_jp, dyz = ey_kp - ey, dzx = ez_ip - ez, dxz = ex - ex_kp, dyx = ey - ey_ip, dxy = ex_jp - ex
    const int i = px + 1, j = py + 1, k = pz + 1;
    const float DB = P.DB;
    const int qx_lo = (i <= P.npml[0][0] - 1) ? i : 0, qx_hi = (i >= P.X + 1 - P.npml[0][1]) ? P.X - i : 0;
    const int qy_lo = (j <= P.npml[1][0] - 1) ? j : 0, qy_hi = (j >= P.Y + 1 - P.npml[1][1]) ? P.Y - j : 0;
    const int qz_lo = (k <= P.npml[2][0] - 1) ? k : 0, qz_hi = (k >= P.Z + 1 - P.npml[2][1]) ? P.Z - k : 0;
    if (qy_lo) hxv = hxv + DB * psi4(P.psi_h[0][1][0], P.psi_h2[0][1][0], store, P.bh[1][0][qy_lo - 1], P.ch[1][0][qy_lo - 1], dzy, P.del[1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]));
    if (qy_hi) hxv = hxv + DB * psi4(P.psi_h[0][1][1], P.psi_h2[0][1][1], store, P.bh[1][1][qy_hi - 1], P.ch[1][1][qy_hi - 1], dzy, P.del[1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]));
    if (qz_lo) hxv = hxv + DB * psi4(P.psi_h[0][2][0], P.psi_h2[0][2][0], store, P.bh[2][0][qz_lo - 1], P.ch[2][0][qz_lo - 1], dyz, P.del[2], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]));
    if (qz_hi) hxv = hxv + DB * psi4(P.psi_h[0][2][1], P.psi_h2[0][2][1], store, P.bh[2][1][qz_hi - 1], P.ch[2][1][qz_hi - 1], dyz, P.del[2], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]));
    if (qx_lo) hyv = hyv + DB * psi4(P.psi_h[1][0][0], P.psi_h2[1][0][0], store, P.bh[0][0][qx_lo - 1], P.ch[0][0][qx_lo - 1], dzx, P.del[0], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]));
    if (qx_hi) hyv = hyv + DB * psi4(P.psi_h[1][0][1], P.psi_h2[1][0][1], store, P.bh[0][1][qx_hi - 1], P.ch[0][1][qx_hi - 1], dzx, P.del[0], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]));
    if (qz_lo) hyv = hyv + DB * psi4(P.psi_h[1][2][0], P.psi_h2[1][2][0], store, P.bh[2][0][qz_lo - 1], P.ch[2][0][qz_lo - 1], dxz, P.del[2], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]));
    if (qz_hi) hyv = hyv + DB * psi4(P.psi_h[1][2][1], P.psi_h2[1][2][1], store, P.bh[2][1][qz_hi - 1], P.ch[2][1][qz_hi - 1], dxz, P.del[2], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]));
    if (qx_lo) hzv = hzv + DB * psi4(P.psi_h[2][0][0], P.psi_h2[2][0][0], store, P.bh[0][0][qx_lo - 1], P.ch[0][0][qx_lo - 1], dyx, P.del[0], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]));
    if (qx_hi) hzv = hzv + DB * psi4(P.psi_h[2][0][1], P.psi_h2[2][0][1], store, P.bh[0][1][qx_hi - 1], P.ch[0][1][qx_hi - 1], dyx, P.del[0], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]));
    if (qy_lo) hzv = hzv + DB * psi4(P.psi_h[2][1][0], P.psi_h2[2][1][0], store, P.bh[1][0][qy_lo - 1], P.ch[1][0][qy_lo - 1], dxy, P.del[1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]));
    if (qy_hi) hzv = hzv + DB * psi4(P.psi_h[2][1][1], P.psi_h2[2][1][1], store, P.bh[1][1][qy_hi - 1], P.ch[1][1][qy_hi - 1], dxy, P.del[1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]));
    return make_float3(hxv, hyv, hzv);
}

// CPML terms of one E cell and component added to its bulk value
__device__ __noinline__ float y4_e_pml(const AemParams& P, int comp, int px, int py, int pz, float e, float gb, float d1,
                                       float d2) {
    const int i = px + 1, j = py + 1, k = pz + 1;
    const int qxl = (i >= 2 && i <= P.npml[0][0]) ? i : 0, qxh = (i >= P.X + 1 - P.npml[0][1] && i <= P.X - 1) ? P.X + 1 - i : 0;
    const int qyl = (j >= 2 && j <= P.npml[1][0]) ? j : 0, qyh = (j >= P.Y + 1 - P.npml[1][1] && j <= P.Y - 1) ? P.Y + 1 - j : 0;
    const int qzl = (k >= 2 && k <= P.npml[2][0]) ? k : 0, qzh = (k >= P.Z + 1 - P.npml[2][1] && k <= P.Z - 1) ? P.Z + 1 - k : 0;
    const int a1 = comp == 0 ? 1 : 0, a2 = comp == 2 ? 1 : 2;
    const int q1l = a1 == 0 ? qxl : qyl, q1h = a1 == 0 ? qxh : qyh;
    const int q2l = a2 == 1 ? qyl : qzl, q2h = a2 == 1 ? qyh : qzh;
    if (q1l) e = e + gb * psi4(P.psi_e[comp][a1][0], P.psi_e[comp][a1][0], true, P.be[a1][0][q1l - 1], P.ce[a1][0][q1l - 1], d1, P.del[a1], psi_idx(P, a1, q1l, px, py, pz, P.npml[a1][0]));
    if (q1h) e = e + gb * psi4(P.psi_e[comp][a1][1], P.psi_e[comp][a1][1], true, P.be[a1][1][q1h - 1], P.ce[a1][1][q1h - 1], d1, P.del[a1], psi_idx(P, a1, q1h, px, py, pz, P.npml[a1][1]));
    if (q2l) e = e + gb * psi4(P.psi_e[comp][a2][0], P.psi_e[comp][a2][0], true, P.be[a2][0][q2l - 1], P.ce[a2][0][q2l - 1], d2, P.del[a2], psi_idx(P, a2, q2l, px, py, pz, P.npml[a2][0]));
    if (q2h) e = e + gb * psi4(P.psi_e[comp][a2][1], P.psi_e[comp][a2][1], true, P.be[a2][1][q2h - 1], P.ce[a2][1][q2h - 1], d2, P.del[a2], psi_idx(P, a2, q2h, px, py, pz, P.npml[a2][1]));
    return e;
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

// H_new of the thread's four cells (row r of the tile, x = xb..xb+3) from
// plane slots E0 (k), E1 (k+1), Ho (H_old k); non-updated cells keep H_old.
// Owned cells (store) also go to H2 / psi_h2.
__device__ inline void y4_h_group(const AemParams& P, const float* E0, const float* E1, const float* Ho, int r, int xi,
                                  int xb, int py, int pz, int hxm, int hym, int hzm, bool store, float hx[4], float hy[4],
                                  float hz[4]) {
    const float* Ex = E0 + (0 * Y4_ER + r) * Y4_EW;
    const float* Ey = E0 + (1 * Y4_ER + r) * Y4_EW;
    const float* Ez = E0 + (2 * Y4_ER + r) * Y4_EW;
    const float4 ex = lds4(Ex + xi), ey = lds4(Ey + xi), ez = lds4(Ez + xi);
    const float4 exj = lds4(Ex + Y4_EW + xi), ezj = lds4(Ez + Y4_EW + xi);
    const float ey4 = Ey[xi + 4], ez4 = Ez[xi + 4];
    const float4 exk = lds4(E1 + (0 * Y4_ER + r) * Y4_EW + xi), eyk = lds4(E1 + (1 * Y4_ER + r) * Y4_EW + xi);
    const float4 h0x = lds4(Ho + (0 * Y4_HR + r) * Y4_HW + xi), h0y = lds4(Ho + (1 * Y4_HR + r) * Y4_HW + xi),
                 h0z = lds4(Ho + (2 * Y4_HR + r) * Y4_HW + xi);
    const float vex[4] = {ex.x, ex.y, ex.z, ex.w}, vey[4] = {ey.x, ey.y, ey.z, ey.w}, vez[4] = {ez.x, ez.y, ez.z, ez.w};
    const float vexj[4] = {exj.x, exj.y, exj.z, exj.w}, vezj[4] = {ezj.x, ezj.y, ezj.z, ezj.w};
    const float veyi[4] = {ey.y, ey.z, ey.w, ey4}, vezi[4] = {ez.y, ez.z, ez.w, ez4};
    const float vexk[4] = {exk.x, exk.y, exk.z, exk.w}, veyk[4] = {eyk.x, eyk.y, eyk.z, eyk.w};
    const float vhx[4] = {h0x.x, h0x.y, h0x.z, h0x.w}, vhy[4] = {h0y.x, h0y.y, h0y.z, h0y.w},
                vhz[4] = {h0z.x, h0z.y, h0z.z, h0z.w};
    const int i0 = xb + 1, j = py + 1, k = pz + 1;
    const bool upd_all = xb + 3 <= hxm && py >= 0 && py <= hym && pz <= hzm;
    const bool no_pml = i0 >= P.npml[0][0] && xb + 4 <= P.X - P.npml[0][1] && j >= P.npml[1][0] &&
                        j <= P.Y - P.npml[1][1] && k >= P.npml[2][0] && k <= P.Z - P.npml[2][1];
    if (upd_all) {
        const float DB = P.DB, dhy = P.den_h[1][j - 1], dhz = P.den_h[2][k - 1];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const float dhx = P.den_h[0][i0 + e - 1];
            hx[e] = vhx[e] + DB * ((vez[e] - vezj[e]) * dhy + (veyk[e] - vey[e]) * dhz);
            hy[e] = vhy[e] + DB * ((vezi[e] - vez[e]) * dhx + (vex[e] - vexk[e]) * dhz);
            hz[e] = vhz[e] + DB * ((vey[e] - veyi[e]) * dhx + (vexj[e] - vex[e]) * dhy);
        }
        if (!no_pml) {
#pragma unroll
            for (int e = 0; e < 4; e++)
            {
                const float3 h = y4_h_pml(P, xb + e, py, pz, vez[e] - vezj[e], veyk[e] - vey[e], vezi[e] - vez[e],
                                          vex[e] - vexk[e], vey[e] - veyi[e], vexj[e] - vex[e], store, hx[e], hy[e], hz[e]);
                hx[e] = h.x; hy[e] = h.y; hz[e] = h.z;
            }
        }
        if (store) {
            const long long c = lin(P, xb, py, pz);
            *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.H2[0]) + c) = make_float4(hx[0], hx[1], hx[2], hx[3]);
            *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.H2[1]) + c) = make_float4(hy[0], hy[1], hy[2], hy[3]);
            *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.H2[2]) + c) = make_float4(hz[0], hz[1], hz[2], hz[3]);
        }
        return;
    }
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int px = xb + e;
        hx[e] = vhx[e]; hy[e] = vhy[e]; hz[e] = vhz[e];
        if (px <= hxm && py >= 0 && py <= hym && pz <= hzm) {
            const float3 h = y4_h_cell(P, px, py, pz, vex[e], vey[e], vez[e], vexj[e], vezj[e], veyi[e], vezi[e], vexk[e],
                                       veyk[e], vhx[e], vhy[e], vhz[e], store);
            hx[e] = h.x; hy[e] = h.y; hz[e] = h.z;
            if (store) {
                const long long c = lin(P, px, py, pz);
                stf4(P.H2[0], c, hx[e]);
                stf4(P.H2[1], c, hy[e]);
                stf4(P.H2[2], c, hz[e]);
            }
        }
    }
}

// the -x halo cell (x0-1, py) of a row: Hy, Hz (never stored)
__device__ __noinline__ float2 y4_h_xhalo(const AemParams& P, const float* E0, const float* E1, const float* Ho, int r,
                                           int x0, int py, int pz, int hxm, int hym, int hzm) {
    const int c3 = 3;  // tile column of x0-1
    const float hyv = Ho[(1 * Y4_HR + r) * Y4_HW + c3];
    const float hzv = Ho[(2 * Y4_HR + r) * Y4_HW + c3];
    const int px = x0 - 1;
    if (px < 0 || px > hxm || py < 0 || py > hym || pz > hzm) return make_float2(hyv, hzv);
    const float* Ex = E0 + (0 * Y4_ER + r) * Y4_EW;
    const float* Ey = E0 + (1 * Y4_ER + r) * Y4_EW;
    const float* Ez = E0 + (2 * Y4_ER + r) * Y4_EW;
    const float3 h = y4_h_cell(P, px, py, pz, Ex[c3], Ey[c3], Ez[c3], Ex[Y4_EW + c3], Ez[Y4_EW + c3], Ey[c3 + 1],
                               Ez[c3 + 1], E1[(0 * Y4_ER + r) * Y4_EW + c3], E1[(1 * Y4_ER + r) * Y4_EW + c3],
                               Ho[(0 * Y4_HR + r) * Y4_HW + c3], hyv, hzv, false);
    return make_float2(h.y, h.z);
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

__global__ void __maxnreg__(112) k_yee4(const __grid_constant__ AemParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    float* Hn = reinterpret_cast<float*>(smem + Y4_OFF_HN);  // [2][9][128]: hx, hz of H_new(k)
    float* gab = Hn + Y4_HN_F;                              // [mat][6]: ga xyz, gb xyz
    const int lane = threadIdx.x, w = threadIdx.y;
    const int tid = lane + 32 * w, nthr = 32 * (Y4_TY + 1);
    const int x0 = blockIdx.x * Y4_TX, y0 = blockIdx.y * Y4_TY;
    const int z0 = blockIdx.z * Y4_ZC, z1 = min(P.SZ, z0 + Y4_ZC);
    const int hxm = P.SX - 2, hym = P.SY - 2, hzm = P.per[2] ? P.SZ - 1 : P.SZ - 2;
    const unsigned FULL = 0xffffffffu;
    for (int q = tid; q < P.nmat * 6; q += nthr) {
        const int m = q / 6, c = q % 6;
        gab[q] = c < 3 ? P.ucoef[m].ga[c] : P.ucoef[m].gb[c - 3];
    }
    auto zw = [&](int p) { return P.per[2] ? (p % P.SZ + P.SZ) % P.SZ : p; };
    auto md = [](int p, int m) { return ((p % m) + m) % m; };
    auto Ew = [&](int p) { return reinterpret_cast<float*>(smem + (size_t)md(p, Y4_ES) * Y4_E_B); };
    auto Hw = [&](int p) { return reinterpret_cast<float*>(smem + Y4_OFF_H + (size_t)md(p, Y4_HS) * Y4_H_B); };
    auto Iw = [&](int p) { return smem + Y4_OFF_I + (size_t)md(p, Y4_IS) * Y4_I_B; };
    auto Es = [&](int p) { return (const float*)Ew(p); };
    auto Hs = [&](int p) { return (const float*)Hw(p); };
    auto Is = [&](int p) { return (const unsigned char*)Iw(p); };

    // this thread's cells: tile row r (0 = the -y halo row), x = xb..xb+3
    const int r = w == Y4_TY ? 0 : w + 1;
    const int py = y0 - 1 + r;
    const int xb = x0 + 4 * lane, xi = 4 * lane + 4, xbi = 4 * lane + 16;
    const bool own = w < Y4_TY && py < P.SY;

    const bool below = P.per[2] || z0 > 0;
    // prologue: E of planes z0-1..z0+1, H and ids of z0-1 and z0
    y4_issue(P, Ew(z0 - 1), Hw(z0 - 1), Iw(z0 - 1), below ? zw(z0 - 1) : -1, x0, y0);
    y4_issue(P, Ew(z0), Hw(z0), Iw(z0), zw(z0), x0, y0);
    y4_issue(P, Ew(z0 + 1), nullptr, nullptr, zw(z0 + 1), x0, y0);
    cp_commit4();
    cp_wait0();
    __syncthreads();
    // H_new(z0-1) of the own cells (the plane below belongs to the chunk underneath)
    float hxp[4] = {0, 0, 0, 0}, hyp[4] = {0, 0, 0, 0};
    if (below && own) {
        float hz_unused[4];
        y4_h_group(P, Es(z0 - 1), Es(z0), Hs(z0 - 1), r, xi, xb, py, zw(z0 - 1), hxm, hym, hzm, false, hxp, hyp, hz_unused);
    }
    const int j = py + 1;
    const float dey = own ? P.den_e[1][j - 1] : 0.0f;

    for (int k = z0; k < z1; k++) {
        const int pz = zw(k);
        // E(k+1), H(k), ids(k) have landed and every thread is done with
        // plane k-1: E(k+2), H(k+1), ids(k+1) reuse the slots of E(k-1),
        // H(k-1), ids(k-2)
        cp_wait0();
        __syncthreads();
        y4_issue(P, Ew(k + 2), nullptr, nullptr, k + 2 <= z1 ? zw(k + 2) : -1, x0, y0);
        y4_issue(P, nullptr, Hw(k + 1), Iw(k + 1), k + 1 < z1 ? zw(k + 1) : -1, x0, y0);
        cp_commit4();

        // ---- H_new(k): own rows, the -y halo row (warp 8), the -x halo cell (lane 0)
        const float* E0 = Es(k);
        float hx[4], hy[4], hz[4];
        if (own || (w == Y4_TY && py >= 0))
            y4_h_group(P, E0, Es(k + 1), Hs(k), r, xi, xb, py, pz, hxm, hym, hzm, own, hx, hy, hz);
        else
            for (int e = 0; e < 4; e++) hx[e] = hy[e] = hz[e] = 0.0f;
        float hy_xh = 0.0f, hz_xh = 0.0f;
        if (lane == 0 && own) {
            const float2 hh = y4_h_xhalo(P, E0, Es(k + 1), Hs(k), r, x0, py, pz, hxm, hym, hzm);
            hy_xh = hh.x; hz_xh = hh.y;
        }
        *reinterpret_cast<float4*>(Hn + (0 * Y4_HR + r) * Y4_TX + 4 * lane) = make_float4(hx[0], hx[1], hx[2], hx[3]);
        *reinterpret_cast<float4*>(Hn + (1 * Y4_HR + r) * Y4_TX + 4 * lane) = make_float4(hz[0], hz[1], hz[2], hz[3]);
        __syncthreads();

        // ---- E_new(k) of the own rows
        if (w < Y4_TY) {
            float hz_im0 = __shfl_up_sync(FULL, hz[3], 1), hy_im0 = __shfl_up_sync(FULL, hy[3], 1);
            if (lane == 0) { hz_im0 = hz_xh; hy_im0 = hy_xh; }
            if (own) {
                const float4 hxj4 = lds4(Hn + (0 * Y4_HR + r - 1) * Y4_TX + 4 * lane);
                const float4 hzj4 = lds4(Hn + (1 * Y4_HR + r - 1) * Y4_TX + 4 * lane);
                const float hxj[4] = {hxj4.x, hxj4.y, hxj4.z, hxj4.w}, hzj[4] = {hzj4.x, hzj4.y, hzj4.z, hzj4.w};
                const float him_z[4] = {hz_im0, hz[0], hz[1], hz[2]}, him_y[4] = {hy_im0, hy[0], hy[1], hy[2]};
                const float4 ex4 = lds4(E0 + (0 * Y4_ER + r) * Y4_EW + xi), ey4 = lds4(E0 + (1 * Y4_ER + r) * Y4_EW + xi),
                             ez4 = lds4(E0 + (2 * Y4_ER + r) * Y4_EW + xi);
                const float vex[4] = {ex4.x, ex4.y, ex4.z, ex4.w}, vey[4] = {ey4.x, ey4.y, ey4.z, ey4.w},
                            vez[4] = {ez4.x, ez4.y, ez4.z, ez4.w};
                const unsigned char* I0 = Is(k);
                const unsigned char* I1 = Is(k - 1);
                const unsigned char* a0 = I0 + r * Y4_IW + xbi;        // plane k, row r
                const unsigned char* a1 = I0 + (r - 1) * Y4_IW + xbi;  // plane k, row r-1
                const unsigned char* b0 = I1 + r * Y4_IW + xbi;        // plane k-1, row r
                const unsigned char* b1 = I1 + (r - 1) * Y4_IW + xbi;  // plane k-1, row r-1
                const unsigned w_a0 = *reinterpret_cast<const unsigned*>(a0), w_a1 = *reinterpret_cast<const unsigned*>(a1);
                const unsigned w_b0 = *reinterpret_cast<const unsigned*>(b0), w_b1 = *reinterpret_cast<const unsigned*>(b1);
                const int kk = pz + 1;
                const float dez = P.den_e[2][kk - 1];
                const bool upd_all = xb >= 1 && xb + 3 <= P.SX - 2 && py >= 1 && py <= P.SY - 2 &&
                                     (P.per[2] || (pz >= 1 && pz <= P.SZ - 2));
                const bool no_pml = xb + 1 > P.npml[0][0] && xb + 4 <= P.X - P.npml[0][1] && j > P.npml[1][0] &&
                                    j < P.Y + 1 - P.npml[1][1] && kk > P.npml[2][0] && kk < P.Z + 1 - P.npml[2][1];
                const unsigned m = a0[0];
                const unsigned rep = m * 0x01010101u;
                const bool uniform = w_a0 == rep && w_a1 == rep && w_b0 == rep && w_b1 == rep && a0[-1] == m &&
                                     a1[-1] == m && b0[-1] == m;
                float ex_n[4], ey_n[4], ez_n[4];
                if (upd_all && uniform) {
                    const float gax = gab[m * 6 + 0], gay = gab[m * 6 + 1], gaz = gab[m * 6 + 2];
                    const float gbx = gab[m * 6 + 3], gby = gab[m * 6 + 4], gbz = gab[m * 6 + 5];
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const float dex = P.den_e[0][xb + e];
                        ex_n[e] = gax * vex[e] + gbx * ((hz[e] - hzj[e]) * dey + (hyp[e] - hy[e]) * dez);
                        ey_n[e] = gay * vey[e] + gby * ((him_z[e] - hz[e]) * dex + (hx[e] - hxp[e]) * dez);
                        ez_n[e] = gaz * vez[e] + gbz * ((hy[e] - him_y[e]) * dex + (hxj[e] - hx[e]) * dey);
                    }
                    if (!no_pml) {
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            ex_n[e] = y4_e_pml(P, 0, xb + e, py, pz, ex_n[e], gbx, hz[e] - hzj[e], hyp[e] - hy[e]);
                            ey_n[e] = y4_e_pml(P, 1, xb + e, py, pz, ey_n[e], gby, him_z[e] - hz[e], hx[e] - hxp[e]);
                            ez_n[e] = y4_e_pml(P, 2, xb + e, py, pz, ez_n[e], gbz, hy[e] - him_y[e], hxj[e] - hx[e]);
                        }
                    }
                    const long long c = lin(P, xb, py, pz);
                    *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.E2[0]) + c) = make_float4(ex_n[0], ex_n[1], ex_n[2], ex_n[3]);
                    *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.E2[1]) + c) = make_float4(ey_n[0], ey_n[1], ey_n[2], ey_n[3]);
                    *reinterpret_cast<float4*>(reinterpret_cast<float*>(P.E2[2]) + c) = make_float4(ez_n[0], ez_n[1], ez_n[2], ez_n[3]);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const int px = xb + e, i = px + 1;
                        if (px >= P.SX) continue;
                        const bool ex_u = px <= P.SX - 2 && py >= 1 && py <= P.SY - 2 && (P.per[2] || (pz >= 1 && pz <= P.SZ - 2));
                        const bool ey_u = px >= 1 && px <= P.SX - 2 && py <= P.SY - 2 && (P.per[2] || (pz >= 1 && pz <= P.SZ - 2));
                        const bool ez_u = px >= 1 && px <= P.SX - 2 && py >= 1 && py <= P.SY - 2 && (P.per[2] || pz <= P.SZ - 2);
                        if (!(ex_u || ey_u || ez_u)) continue;
                        const bool unavg = i == 1 || j == 1 || (!P.per[2] && kk == 1);
                        const int idc = unavg ? 0 : a0[e], idx_ = unavg ? 0 : a0[e - 1], idy_ = unavg ? 0 : a1[e],
                                  idxy = unavg ? 0 : a1[e - 1];
                        const int pdc = unavg ? 0 : b0[e], pdx = unavg ? 0 : b0[e - 1], pdy = unavg ? 0 : b1[e];
                        const float dex = P.den_e[0][i - 1];
                        const long long c = lin(P, px, py, pz);
                        if (ex_u) stf4(P.E2[0], c, y4_e_comp(P, gab, 0, px, py, pz, vex[e], hz[e] - hzj[e], hyp[e] - hy[e], dey, dez, idc, idy_, pdc, pdy));
                        if (ey_u) stf4(P.E2[1], c, y4_e_comp(P, gab, 1, px, py, pz, vey[e], him_z[e] - hz[e], hx[e] - hxp[e], dex, dez, idc, idx_, pdc, pdx));
                        if (ez_u) stf4(P.E2[2], c, y4_e_comp(P, gab, 2, px, py, pz, vez[e], hy[e] - him_y[e], hxj[e] - hx[e], dex, dey, idc, idx_, idy_, idxy));
                    }
                }
            }
        }
#pragma unroll
        for (int e = 0; e < 4; e++) { hxp[e] = hx[e]; hyp[e] = hy[e]; }
    }
    cp_wait0();  // no copy may still target this CTA's shared memory at exit
}

int launch_yee4(const AemParams& P, cudaStream_t s) {
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        cudaFuncSetAttribute(k_yee4, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Y4_SMEM);
        attr_set[dev] = true;
    }
    // the last position of a non-periodic axis is never updated: no tile for it
    const int ux = P.SX - 1, uy = P.SY - 1, uz = P.per[2] ? P.SZ : P.SZ - 1;
    dim3 blk(32, Y4_TY + 1), grd((ux + Y4_TX - 1) / Y4_TX, (uy + Y4_TY - 1) / Y4_TY, (uz + Y4_ZC - 1) / Y4_ZC);
    k_yee4<<<grd, blk, Y4_SMEM, s>>>(P);
    return 1;
}

}  // namespace aem
