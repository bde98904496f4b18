// aem_yee.cu -- fused H+E time step (FP32, standard solver).
//
// One kernel advances H^{n-1/2} -> H^{n+1/2} and E^n -> E^{n+1} in a single
// pass over the grid, so each field value is read once and written once per
// step (49 B per cell with the material byte) instead of the >= 73 B of a
// separate H pass and E pass.  Same arithmetic, statement for statement, as
// k_update_h / k_update_e (bulk curl fdtd_solver.f90:4442-4484 and
// :5667-5710, CPML :5227-5375 and :6522-6670, periodic wrap :5377-5433 and
// :6672-6806), so the fields are bit-identical to the two-kernel path.
//
// Layout: a CTA is 32 x 8 threads, one storage x-row per warp, and marches z
// over a chunk of planes.  At plane k a thread
//   1. computes H_new(k) of its cell from E_old (k and k+1) -- the +x
//      neighbour comes from the next lane (shuffle), the +y neighbour from
//      the next warp (shared memory), the +z one is next plane's own load;
//   2. computes E_new(k) from H_new(k) (own, -x by shuffle, -y by shared
//      memory) and H_new(k-1) (own, kept from the previous plane).
// The -x column of lane 0 and the -y row of warp 0 belong to other CTAs,
// which may already have stored their new values, so fields and H-psi are
// double-buffered (read E/H/psi_h, write E2/H2/psi_h2; the host swaps) and
// lane 0 / warp 0 recompute those halo H values from the old buffers with
// the same expressions (bit-identical, never stored).  A chunk that does not
// start at z = 0 recomputes H_new of the plane below it the same way.
//
// Used when the deck has no TF/SF source, sheets, Drude poles, gridded
// ports or kmax (those keep the two-kernel path).
#include <cstdlib>
#include <cstring>

#include "aem_dev.cuh"
#include "aem_kernels.h"

namespace aem {

constexpr int YEE_TY = 8;   // rows (warps) per CTA
constexpr int YEE_ZC = 64;  // planes per z chunk

__device__ inline float ldf(const void* b, long long i) { return reinterpret_cast<const float*>(b)[i]; }
__device__ inline void stf(void* b, long long i, float v) { reinterpret_cast<float*>(b)[i] = v; }

// E values one H cell needs (old fields)
struct HNb {
    float ex, ey, ez;      // at the cell
    float ex_jp, ez_jp;    // at y+1
    float ey_ip, ez_ip;    // at x+1
    float ex_kp, ey_kp;    // at z+1
};

// CPML psi update psi_new = b psi_old + c diff / dl (ref :5234 / :6529),
// read from `rd`, written to `wr` when `store`
__device__ inline float psi_term(const void* rd, void* wr, bool store, float b, float c, float diff, float dl,
                                 long long q) {
    const float nw = b * ldf(rd, q) + cpml_div(c * diff, dl);
    if (store) stf(wr, q, nw);
    return nw;
}

// H_new of the components in `mask` (1 Hx, 2 Hy, 4 Hz) of cell (px,py,pz),
// as k_update_h computes it (no sheets / TF/SF on this path)
__device__ inline void h_cell(const AemParams& P, int px, int py, int pz, const HNb& e, int mask, bool store,
                              float& hxv, float& hyv, float& hzv) {
    const int i = px + 1, j = py + 1, k = pz + 1;
    const float DB = P.DB;
    const float dhx = P.den_h[0][i - 1], dhy = P.den_h[1][j - 1], dhz = P.den_h[2][k - 1];
    const long long c = lin(P, px, py, pz);
    const int qx_lo = (i <= P.npml[0][0] - 1) ? i : 0, qx_hi = (i >= P.X + 1 - P.npml[0][1]) ? P.X - i : 0;
    const int qy_lo = (j <= P.npml[1][0] - 1) ? j : 0, qy_hi = (j >= P.Y + 1 - P.npml[1][1]) ? P.Y - j : 0;
    const int qz_lo = (k <= P.npml[2][0] - 1) ? k : 0, qz_hi = (k >= P.Z + 1 - P.npml[2][1]) ? P.Z - k : 0;
    if (mask & 1) {
        hxv = ldf(P.H[0], c) + DB * ((e.ez - e.ez_jp) * dhy + (e.ey_kp - e.ey) * dhz);
        if (qy_lo) hxv = hxv + DB * psi_term(P.psi_h[0][1][0], P.psi_h2[0][1][0], store, P.bh[1][0][qy_lo - 1], P.ch[1][0][qy_lo - 1], e.ez - e.ez_jp, P.del[1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]));
        if (qy_hi) hxv = hxv + DB * psi_term(P.psi_h[0][1][1], P.psi_h2[0][1][1], store, P.bh[1][1][qy_hi - 1], P.ch[1][1][qy_hi - 1], e.ez - e.ez_jp, P.del[1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]));
        if (qz_lo) hxv = hxv + DB * psi_term(P.psi_h[0][2][0], P.psi_h2[0][2][0], store, P.bh[2][0][qz_lo - 1], P.ch[2][0][qz_lo - 1], e.ey_kp - e.ey, P.del[2], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]));
        if (qz_hi) hxv = hxv + DB * psi_term(P.psi_h[0][2][1], P.psi_h2[0][2][1], store, P.bh[2][1][qz_hi - 1], P.ch[2][1][qz_hi - 1], e.ey_kp - e.ey, P.del[2], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]));
    }
    if (mask & 2) {
        hyv = ldf(P.H[1], c) + DB * ((e.ez_ip - e.ez) * dhx + (e.ex - e.ex_kp) * dhz);
        if (qx_lo) hyv = hyv + DB * psi_term(P.psi_h[1][0][0], P.psi_h2[1][0][0], store, P.bh[0][0][qx_lo - 1], P.ch[0][0][qx_lo - 1], e.ez_ip - e.ez, P.del[0], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]));
        if (qx_hi) hyv = hyv + DB * psi_term(P.psi_h[1][0][1], P.psi_h2[1][0][1], store, P.bh[0][1][qx_hi - 1], P.ch[0][1][qx_hi - 1], e.ez_ip - e.ez, P.del[0], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]));
        if (qz_lo) hyv = hyv + DB * psi_term(P.psi_h[1][2][0], P.psi_h2[1][2][0], store, P.bh[2][0][qz_lo - 1], P.ch[2][0][qz_lo - 1], e.ex - e.ex_kp, P.del[2], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]));
        if (qz_hi) hyv = hyv + DB * psi_term(P.psi_h[1][2][1], P.psi_h2[1][2][1], store, P.bh[2][1][qz_hi - 1], P.ch[2][1][qz_hi - 1], e.ex - e.ex_kp, P.del[2], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]));
    }
    if (mask & 4) {
        hzv = ldf(P.H[2], c) + DB * ((e.ey - e.ey_ip) * dhx + (e.ex_jp - e.ex) * dhy);
        if (qx_lo) hzv = hzv + DB * psi_term(P.psi_h[2][0][0], P.psi_h2[2][0][0], store, P.bh[0][0][qx_lo - 1], P.ch[0][0][qx_lo - 1], e.ey - e.ey_ip, P.del[0], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]));
        if (qx_hi) hzv = hzv + DB * psi_term(P.psi_h[2][0][1], P.psi_h2[2][0][1], store, P.bh[0][1][qx_hi - 1], P.ch[0][1][qx_hi - 1], e.ey - e.ey_ip, P.del[0], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]));
        if (qy_lo) hzv = hzv + DB * psi_term(P.psi_h[2][1][0], P.psi_h2[2][1][0], store, P.bh[1][0][qy_lo - 1], P.ch[1][0][qy_lo - 1], e.ex_jp - e.ex, P.del[1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]));
        if (qy_hi) hzv = hzv + DB * psi_term(P.psi_h[2][1][1], P.psi_h2[2][1][1], store, P.bh[1][1][qy_hi - 1], P.ch[1][1][qy_hi - 1], e.ex_jp - e.ex, P.del[1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]));
    }
}

// Ga/Gb of an E edge from its four cells (ids in the reference's order,
// ref :2516-2527); no sheet or Drude terms on this path
__device__ inline void edge_gagb(const AemParams& P, int c, int i0, int i1, int i2, int i3, float& ga, float& gb) {
    if (i0 == i1 && i0 == i2 && i0 == i3) {
        ga = P.ucoef[i0].ga[c];
        gb = P.ucoef[i0].gb[c];
        return;
    }
    const AemMaterial *m0 = P.mat + i0, *m1 = P.mat + i1, *m2 = P.mat + i2, *m3 = P.mat + i3;
    const float e = (m0->eps[c] + m1->eps[c] + m2->eps[c] + m3->eps[c]) / 4.0f;
    const float s = (m0->sig[c] + m1->sig[c] + m2->sig[c] + m3->sig[c]) / 4.0f;
    const float tp = 0.0f;
    ga = d_ga(s + tp, e, P.dt);
    gb = d_gb(s + tp, e, P.dt);
}

__global__ void __launch_bounds__(256) k_yee(const __grid_constant__ AemParams P) {
    __shared__ float sEx[YEE_TY][32], sEz[YEE_TY][32], sHx[YEE_TY][32], sHz[YEE_TY][32];
    const int lane = threadIdx.x, ty = threadIdx.y;
    const int px = blockIdx.x * 32 + lane, py = blockIdx.y * YEE_TY + ty;
    const bool live = px < P.SX && py < P.SY;
    const int z0 = blockIdx.z * YEE_ZC, z1 = min(P.SZ, z0 + YEE_ZC);
    const unsigned FULL = 0xffffffffu;

    // neighbour positions (x/y wrap on periodic axes; -1 / S off the grid)
    const int pxn = (px + 1 == P.SX && P.per[0]) ? 0 : px + 1;
    const int pyn = (py + 1 == P.SY && P.per[1]) ? 0 : py + 1;
    // +x / +y neighbours come from the next lane / warp unless they wrap or
    // lie outside this CTA
    const bool xn_local = lane < 31 && pxn == px + 1;
    const bool yn_local = ty < YEE_TY - 1 && pyn == py + 1;
    int pxd = (px == 0 && P.per[0]) ? P.SX - 1 : px - 1;
    int pyd = (py == 0 && P.per[1]) ? P.SY - 1 : py - 1;
    // update ranges (k_update_h / k_update_e)
    const int hxm = P.per[0] ? P.SX - 1 : P.SX - 2, hym = P.per[1] ? P.SY - 1 : P.SY - 2, hzm = P.per[2] ? P.SZ - 1 : P.SZ - 2;
    const bool h_xy = live && px <= hxm && py <= hym;
    auto upd = [&](int a, int p, bool normal) {
        const int S = a == 0 ? P.SX : a == 1 ? P.SY : P.SZ;
        if (P.per[a]) return true;
        return normal ? (p <= S - 2) : (p >= 1 && p <= S - 2);
    };
    const bool ex_xy = live && upd(0, px, true) && upd(1, py, false);
    const bool ey_xy = live && upd(0, px, false) && upd(1, py, true);
    const bool ez_xy = live && upd(0, px, false) && upd(1, py, false);
    // halo cells this thread recomputes: lane 0 the -x column (Hy, Hz),
    // warp 0 the -y row (Hx, Hz); only where an E update reads them
    const bool hx_halo = lane == 0 && live && pxd >= 0 && (ey_xy || ez_xy) && pxd <= hxm && py <= hym;
    const bool hy_halo = ty == 0 && live && pyd >= 0 && (ex_xy || ez_xy) && px <= hxm && pyd <= hym;
    if (pxd < 0) pxd = 0;  // only read by components not updated here
    if (pyd < 0) pyd = 0;
    const int i = px + 1, j = py + 1;
    const float dex = live ? P.den_e[0][i - 1] : 0.0f, dey = live ? P.den_e[1][j - 1] : 0.0f;
    const int qxl = (i >= 2 && i <= P.npml[0][0]) ? i : 0, qxh = (i >= P.X + 1 - P.npml[0][1] && i <= P.X - 1) ? P.X + 1 - i : 0;
    const int qyl = (j >= 2 && j <= P.npml[1][0]) ? j : 0, qyh = (j >= P.Y + 1 - P.npml[1][1] && j <= P.Y - 1) ? P.Y + 1 - j : 0;
    const bool xy_unavg = (!P.per[0] && i == 1) || (!P.per[1] && j == 1);

    auto zwrap_up = [&](int pz) { return (pz + 1 == P.SZ && P.per[2]) ? 0 : pz + 1; };
    auto zwrap_dn = [&](int pz) { return (pz == 0 && P.per[2]) ? P.SZ - 1 : pz - 1; };
    // cell ids of the four (x,y) corners of plane pz: own, -x, -y, -x-y
    auto load_ids = [&](int pz, int& ic, int& ixd, int& iyd, int& ixyd) {
        ic = live ? P.cell[lin(P, px, py, pz)] : 0;
        iyd = live ? P.cell[lin(P, px, pyd, pz)] : 0;
        ixd = live ? P.cell[lin(P, pxd, py, pz)] : 0;
        ixyd = live ? P.cell[lin(P, pxd, pyd, pz)] : 0;
    };

    // E_old at the first plane, H_new of the plane below the chunk
    float ex = 0.0f, ey = 0.0f, ez = 0.0f, hxp = 0.0f, hyp = 0.0f;
    int pic = 0, pixd = 0, piyd = 0, pixyd = 0;  // ids of plane pz-1
    if (live) {
        const long long c = lin(P, px, py, z0);
        ex = ldf(P.E[0], c); ey = ldf(P.E[1], c); ez = ldf(P.E[2], c);
    }
    {
        const int pzd = zwrap_dn(z0);
        if (pzd >= 0) {
            load_ids(pzd, pic, pixd, piyd, pixyd);
            if (h_xy && pzd <= hzm) {
                HNb e;
                const long long c = lin(P, px, py, pzd);
                e.ex = ldf(P.E[0], c); e.ey = ldf(P.E[1], c); e.ez = ldf(P.E[2], c);
                e.ex_jp = ldf(P.E[0], lin(P, px, pyn, pzd)); e.ez_jp = ldf(P.E[2], lin(P, px, pyn, pzd));
                e.ey_ip = ldf(P.E[1], lin(P, pxn, py, pzd)); e.ez_ip = ldf(P.E[2], lin(P, pxn, py, pzd));
                e.ex_kp = ex; e.ey_kp = ey;
                float hz_unused;
                h_cell(P, px, py, pzd, e, 3, false, hxp, hyp, hz_unused);
            } else if (live) {
                const long long c = lin(P, px, py, pzd);
                hxp = ldf(P.H[0], c); hyp = ldf(P.H[1], c);
            }
        }
    }

    for (int pz = z0; pz < z1; pz++) {
        const int k = pz + 1;
        const int pzn = zwrap_up(pz);
        const bool h_here = h_xy && pz <= hzm;
        // E_old of the next plane (own cell), this plane's +z neighbour
        float exn = 0.0f, eyn = 0.0f, ezn = 0.0f;
        if (live && pzn < P.SZ) {
            const long long cn = lin(P, px, py, pzn);
            exn = ldf(P.E[0], cn); eyn = ldf(P.E[1], cn); ezn = ldf(P.E[2], cn);
        }
        int ic, ixd, iyd, ixyd;
        load_ids(pz, ic, ixd, iyd, ixyd);
        sEx[ty][lane] = ex;
        sEz[ty][lane] = ez;
        // +x neighbour from the next lane (lane 31 and wrapped ones load it)
        float ey_ip = __shfl_down_sync(FULL, ey, 1), ez_ip = __shfl_down_sync(FULL, ez, 1);
        if (!xn_local && h_here) {
            const long long c = lin(P, pxn, py, pz);
            ey_ip = ldf(P.E[1], c); ez_ip = ldf(P.E[2], c);
        }
        __syncthreads();

        // ---- H_new(pz) of the own cell
        float hx = 0.0f, hy = 0.0f, hz = 0.0f;
        const long long c = lin(P, px, py, pz);
        if (h_here) {
            HNb e;
            e.ex = ex; e.ey = ey; e.ez = ez;
            if (yn_local) { e.ex_jp = sEx[ty + 1][lane]; e.ez_jp = sEz[ty + 1][lane]; }
            else { const long long cj = lin(P, px, pyn, pz); e.ex_jp = ldf(P.E[0], cj); e.ez_jp = ldf(P.E[2], cj); }
            e.ey_ip = ey_ip; e.ez_ip = ez_ip;
            e.ex_kp = exn; e.ey_kp = eyn;
            h_cell(P, px, py, pz, e, 7, true, hx, hy, hz);
        } else if (live) {
            hx = ldf(P.H[0], c); hy = ldf(P.H[1], c); hz = ldf(P.H[2], c);
        }
        // ---- halo H of the -x column (lane 0): Hy, Hz at (pxd, py, pz)
        float hy_xh = 0.0f, hz_xh = 0.0f;
        if (lane == 0 && live) {
            if (hx_halo && pz <= hzm) {
                HNb e;
                const long long cd = lin(P, pxd, py, pz);
                e.ex = ldf(P.E[0], cd); e.ey = ldf(P.E[1], cd); e.ez = ldf(P.E[2], cd);
                e.ex_jp = ldf(P.E[0], lin(P, pxd, pyn, pz)); e.ez_jp = 0.0f;
                e.ey_ip = ey; e.ez_ip = ez;
                e.ex_kp = ldf(P.E[0], lin(P, pxd, py, pzn)); e.ey_kp = 0.0f;
                float hx_unused;
                h_cell(P, pxd, py, pz, e, 6, false, hx_unused, hy_xh, hz_xh);
            } else {
                const long long cd = lin(P, pxd, py, pz);
                hy_xh = ldf(P.H[1], cd); hz_xh = ldf(P.H[2], cd);
            }
        }
        // ---- halo H of the -y row (warp 0): Hx, Hz at (px, pyd, pz)
        float hx_yh = 0.0f, hz_yh = 0.0f;
        {
            // the -y row's +x neighbour Ey comes from the next lane as well
            float ey_d = 0.0f, ex_d = 0.0f, ez_d = 0.0f;
            const bool need = ty == 0 && hy_halo && pz <= hzm;
            if (ty == 0 && live) {
                const long long cd = lin(P, px, pyd, pz);
                ex_d = ldf(P.E[0], cd); ey_d = ldf(P.E[1], cd); ez_d = ldf(P.E[2], cd);
            }
            float ey_d_ip = __shfl_down_sync(FULL, ey_d, 1);
            if (need) {
                if (!xn_local) ey_d_ip = ldf(P.E[1], lin(P, pxn, pyd, pz));
                HNb e;
                e.ex = ex_d; e.ey = ey_d; e.ez = ez_d;
                e.ex_jp = ex; e.ez_jp = ez;  // the own row is the -y row's +y neighbour
                e.ey_ip = ey_d_ip; e.ez_ip = 0.0f;
                e.ex_kp = 0.0f; e.ey_kp = ldf(P.E[1], lin(P, px, pyd, pzn));
                float hy_unused;
                h_cell(P, px, pyd, pz, e, 5, false, hx_yh, hy_unused, hz_yh);
            } else if (ty == 0 && live) {
                const long long cd = lin(P, px, pyd, pz);
                hx_yh = ldf(P.H[0], cd); hz_yh = ldf(P.H[2], cd);
            }
        }
        sHx[ty][lane] = hx;
        sHz[ty][lane] = hz;
        __syncthreads();

        // ---- E_new(pz) of the own cell
        const bool ex_u = ex_xy && upd(2, pz, false), ey_u = ey_xy && upd(2, pz, false), ez_u = ez_xy && upd(2, pz, true);
        float hz_im = __shfl_up_sync(FULL, hz, 1), hy_im = __shfl_up_sync(FULL, hy, 1);
        if (lane == 0) { hz_im = hz_xh; hy_im = hy_xh; }
        const float hz_jm = ty > 0 ? sHz[ty - 1][lane] : hz_yh;
        const float hx_jm = ty > 0 ? sHx[ty - 1][lane] : hx_yh;
        if (ex_u || ey_u || ez_u) {
            const float dez = P.den_e[2][k - 1];
            const bool unavg = xy_unavg || (!P.per[2] && k == 1);
            const int qzl = (k >= 2 && k <= P.npml[2][0]) ? k : 0, qzh = (k >= P.Z + 1 - P.npml[2][1] && k <= P.Z - 1) ? P.Z + 1 - k : 0;
            const int idc = unavg ? 0 : ic, idx_ = unavg ? 0 : ixd, idy_ = unavg ? 0 : iyd, idxy = unavg ? 0 : ixyd;
            const int pdc = unavg ? 0 : pic, pdx = unavg ? 0 : pixd, pdy = unavg ? 0 : piyd;
            if (ex_u) {
                const float d1 = hz - hz_jm, d2 = hyp - hy;
                const float curl = d1 * dey + d2 * dez;
                float ga, gb;
                edge_gagb(P, 0, idc, idy_, pdc, pdy, ga, gb);
                float e = ga * ex + gb * curl;
                if (qyl) e = e + gb * psi_term(P.psi_e[0][1][0], P.psi_e[0][1][0], true, P.be[1][0][qyl - 1], P.ce[1][0][qyl - 1], d1, P.del[1], psi_idx(P, 1, qyl, px, py, pz, P.npml[1][0]));
                if (qyh) e = e + gb * psi_term(P.psi_e[0][1][1], P.psi_e[0][1][1], true, P.be[1][1][qyh - 1], P.ce[1][1][qyh - 1], d1, P.del[1], psi_idx(P, 1, qyh, px, py, pz, P.npml[1][1]));
                if (qzl) e = e + gb * psi_term(P.psi_e[0][2][0], P.psi_e[0][2][0], true, P.be[2][0][qzl - 1], P.ce[2][0][qzl - 1], d2, P.del[2], psi_idx(P, 2, qzl, px, py, pz, P.npml[2][0]));
                if (qzh) e = e + gb * psi_term(P.psi_e[0][2][1], P.psi_e[0][2][1], true, P.be[2][1][qzh - 1], P.ce[2][1][qzh - 1], d2, P.del[2], psi_idx(P, 2, qzh, px, py, pz, P.npml[2][1]));
                stf(P.E2[0], c, e);
            }
            if (ey_u) {
                const float d1 = hz_im - hz, d2 = hx - hxp;
                const float curl = d1 * dex + d2 * dez;
                float ga, gb;
                edge_gagb(P, 1, idc, idx_, pdc, pdx, ga, gb);
                float e = ga * ey + gb * curl;
                if (qxl) e = e + gb * psi_term(P.psi_e[1][0][0], P.psi_e[1][0][0], true, P.be[0][0][qxl - 1], P.ce[0][0][qxl - 1], d1, P.del[0], psi_idx(P, 0, qxl, px, py, pz, P.npml[0][0]));
                if (qxh) e = e + gb * psi_term(P.psi_e[1][0][1], P.psi_e[1][0][1], true, P.be[0][1][qxh - 1], P.ce[0][1][qxh - 1], d1, P.del[0], psi_idx(P, 0, qxh, px, py, pz, P.npml[0][1]));
                if (qzl) e = e + gb * psi_term(P.psi_e[1][2][0], P.psi_e[1][2][0], true, P.be[2][0][qzl - 1], P.ce[2][0][qzl - 1], d2, P.del[2], psi_idx(P, 2, qzl, px, py, pz, P.npml[2][0]));
                if (qzh) e = e + gb * psi_term(P.psi_e[1][2][1], P.psi_e[1][2][1], true, P.be[2][1][qzh - 1], P.ce[2][1][qzh - 1], d2, P.del[2], psi_idx(P, 2, qzh, px, py, pz, P.npml[2][1]));
                stf(P.E2[1], c, e);
            }
            if (ez_u) {
                const float d1 = hy - hy_im, d2 = hx_jm - hx;
                const float curl = d1 * dex + d2 * dey;
                float ga, gb;
                edge_gagb(P, 2, idc, idx_, idy_, idxy, ga, gb);
                float e = ga * ez + gb * curl;
                if (qxl) e = e + gb * psi_term(P.psi_e[2][0][0], P.psi_e[2][0][0], true, P.be[0][0][qxl - 1], P.ce[0][0][qxl - 1], d1, P.del[0], psi_idx(P, 0, qxl, px, py, pz, P.npml[0][0]));
                if (qxh) e = e + gb * psi_term(P.psi_e[2][0][1], P.psi_e[2][0][1], true, P.be[0][1][qxh - 1], P.ce[0][1][qxh - 1], d1, P.del[0], psi_idx(P, 0, qxh, px, py, pz, P.npml[0][1]));
                if (qyl) e = e + gb * psi_term(P.psi_e[2][1][0], P.psi_e[2][1][0], true, P.be[1][0][qyl - 1], P.ce[1][0][qyl - 1], d2, P.del[1], psi_idx(P, 1, qyl, px, py, pz, P.npml[1][0]));
                if (qyh) e = e + gb * psi_term(P.psi_e[2][1][1], P.psi_e[2][1][1], true, P.be[1][1][qyh - 1], P.ce[1][1][qyh - 1], d2, P.del[1], psi_idx(P, 1, qyh, px, py, pz, P.npml[1][1]));
                stf(P.E2[2], c, e);
            }
        }
        if (h_here) {
            stf(P.H2[0], c, hx);
            stf(P.H2[1], c, hy);
            stf(P.H2[2], c, hz);
        }
        // carry to the next plane
        hxp = hx; hyp = hy;
        ex = exn; ey = eyn; ez = ezn;
        pic = ic; pixd = ixd; piyd = iyd; pixyd = ixyd;
    }
}

// ---------------------------------------------------------------------------
bool yee_fused_ok(const AemParams& P, int gridded_ports) {
    return !P.kmax && !P.tfsf_on && !P.mirror_on && P.nsheet == 0 && P.npoles == 0 && !P.has_drude &&
           !P.kmax_mode_TE && !P.kmax_mode_TM && gridded_ports == 0;
}

int launch_yee(const AemParams& P, cudaStream_t s) {
    // grids without x/y periodicity: the TMA-fed 4-cells-per-thread kernel
    if (!P.per[0] && !P.per[1]) return launch_yee4(P, s);
    dim3 blk(32, YEE_TY), grd((P.SX + 31) / 32, (P.SY + YEE_TY - 1) / YEE_TY, (P.SZ + YEE_ZC - 1) / YEE_ZC);
    k_yee<<<grd, blk, 0, s>>>(P);
    return 1;
}

}  // namespace aem
