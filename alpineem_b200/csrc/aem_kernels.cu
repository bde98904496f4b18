// aem_kernels.cu -- the per-step field updates on sm_100a.
//
// Two bandwidth-bound kernels per time step, each a 2.5D march along z over
// (32 x 8)-thread column tiles:
//   k_update_h : H^{n+1/2} from E^n  -- bulk curl (fdtd_solver.f90:4442-4484),
//                Smith-Maloney sheet terms (:4486-4554), TF/SF or kmax plane
//                source (:4558-4794), CPML psi (:5227-5375), PBC (:5377-5433)
//                by periodic indexing
//   k_update_e : E^{n+1} from H     -- bulk update with per-cell material IDs
//                (:5667-5710), sheet sub-cell field (:5712-5780), Drude ADE
//                (:5782-5854), TF/SF or kmax plane source (:5857-6117), CPML
//                psi (:6522-6670), PBC (:6672-6806) by periodic indexing
// The ports, far-field and output taps run as small kernels in
// aem_aux.cu.  Every correction is applied in the reference's statement
// order; built with -fmad=false so the FP32 results round like the
// reference's expressions.
#include "aem_dev.cuh"
#include "aem_kernels.h"

namespace aem {

template <typename T>
__device__ inline T ld(const void* base, long long i) {
    return reinterpret_cast<const T*>(base)[i];
}
template <typename T>
__device__ inline void st(void* base, long long i, T v) {
    reinterpret_cast<T*>(base)[i] = v;
}

// read a neighbour that may sit across a periodic boundary (Bloch phase
// exp(-ikL) when stepping past the last position)
template <typename T>
__device__ inline T ld_up(const AemParams& P, const void* base, long long i, bool wrapped, int axis) {
    T v = ld<T>(base, i);
    return wrapped ? bloch<T>(v, P, axis, -1) : v;
}
template <typename T>
__device__ inline T ld_dn(const AemParams& P, const void* base, long long i, bool wrapped, int axis) {
    T v = ld<T>(base, i);
    return wrapped ? bloch<T>(v, P, axis, +1) : v;
}

// CPML psi update and add-on, ref :5234-5236 (H) / :6529-6531 (E)
template <typename T>
__device__ inline T cpml_term(const AemParams& P, void* psi, float b, float c, T diff, float dl, long long q) {
    T old = ld<T>(psi, q);
    T nw = b * old + cpml_div(c * diff, dl);
    st<T>(psi, q, nw);
    return nw;
}

// z planes per CTA of the two-kernel path (P.zch_h / P.zch_e) and rows per
// CTA (P.ty_h / P.ty_e, 32 columns each): z chunks let a grid narrow in x
// and y (a kmax unit cell) spread over every SM.  The default is 16 planes
// of 8 rows; Solver::autotune times the candidates on a run's own steps.
constexpr int UPD_ZCH = 16, UPD_TY = 8;

// TF/SF corrections of one H position (FP32 runs), ref :4627-4794
// (incident then mirrored); i, j, k reference indices
__device__ __forceinline__ void tfsf_h(const AemParams& P, int i, int j, int k, float cntH, float& hxv, float& hyv,
                                      float& hzv) {
    if (P.tfsf_on) {  // TF/SF faces, ref :4627-4794 (incident then mirrored)
        const int xl = P.lo[0], xh = P.hi[0], yl = P.lo[1], yh = P.hi[1], zl = P.lo[2], zh = P.hi[2];
        for (int m = 0; m <= P.mirror_on; m++) {
            const float wEx = P.WE[m][0], wEy = P.WE[m][1], wEz = P.WE[m][2];
            if (!P.per[1]) {
                const float cf_ = P.coef_h[1];
                if (j == yl - 1 || j == yh) {
                    const float yy = (float)(j == yh ? yh : yl), w = j == yh ? P.wall_hi[1] : P.wall_lo[1];
                    const float sg = j == yh ? 1.0f : -1.0f;
                    if (k >= zl && k <= zh && i >= xl && i <= xh - 1 + P.per[0])
                        hzv = sg > 0 ? hzv + cf_ * d_inc(P, m, wEx, (float)i + 0.5f, yy, (float)k, cntH) * w
                                     : hzv - cf_ * d_inc(P, m, wEx, (float)i + 0.5f, yy, (float)k, cntH) * w;
                    if (k >= zl && k <= zh - 1 + P.per[2] && i >= xl && i <= xh)
                        hxv = sg > 0 ? hxv - cf_ * d_inc(P, m, wEz, (float)i, yy, (float)k + 0.5f, cntH) * w
                                     : hxv + cf_ * d_inc(P, m, wEz, (float)i, yy, (float)k + 0.5f, cntH) * w;
                }
            }
            if (!P.per[2]) {
                const float cf_ = P.coef_h[2];
                if (k == zl - 1 || k == zh) {
                    const float zz = (float)(k == zh ? zh : zl), w = k == zh ? P.wall_hi[2] : P.wall_lo[2];
                    const bool hiface = k == zh;
                    if (j >= yl && j <= yh && i >= xl && i <= xh - 1 + P.per[0])
                        hyv = hiface ? hyv - cf_ * d_inc(P, m, wEx, (float)i + 0.5f, (float)j, zz, cntH) * w
                                     : hyv + cf_ * d_inc(P, m, wEx, (float)i + 0.5f, (float)j, zz, cntH) * w;
                    if (j >= yl && j <= yh - 1 + P.per[1] && i >= xl && i <= xh)
                        hxv = hiface ? hxv + cf_ * d_inc(P, m, wEy, (float)i, (float)j + 0.5f, zz, cntH) * w
                                     : hxv - cf_ * d_inc(P, m, wEy, (float)i, (float)j + 0.5f, zz, cntH) * w;
                }
            }
            if (!P.per[0]) {
                const float cf_ = P.coef_h[0];
                if (i == xl - 1 || i == xh) {
                    const float xx = (float)(i == xh ? xh : xl), w = i == xh ? P.wall_hi[0] : P.wall_lo[0];
                    const bool hiface = i == xh;
                    if (k >= zl && k <= zh && j >= yl && j <= yh - 1 + P.per[1])
                        hzv = hiface ? hzv - cf_ * d_inc(P, m, wEy, xx, (float)j + 0.5f, (float)k, cntH) * w
                                     : hzv + cf_ * d_inc(P, m, wEy, xx, (float)j + 0.5f, (float)k, cntH) * w;
                    if (k >= zl && k <= zh - 1 + P.per[2] && j >= yl && j <= yh)
                        hyv = hiface ? hyv + cf_ * d_inc(P, m, wEz, xx, (float)j, (float)k + 0.5f, cntH) * w
                                     : hyv - cf_ * d_inc(P, m, wEz, xx, (float)j, (float)k + 0.5f, cntH) * w;
                }
            }
        }
    }
}

// TF/SF correction of E component comp (FP32 runs), ref :5950-6117; ri, rj,
// rk the component's representative reference indices
__device__ __forceinline__ void tfsf_e(const AemParams& P, int comp, int ri, int rj, int rk, float cntE, float& e) {
    if (P.tfsf_on) {  // TF/SF faces, ref :5950-6117
        const int xl = P.lo[0], xh = P.hi[0], yl = P.lo[1], yh = P.hi[1], zl = P.lo[2], zh = P.hi[2];
        const int pbx = P.per[0], pby = P.per[1], pbz = P.per[2];
        for (int m = 0; m <= P.mirror_on; m++) {
            const float wHx = P.WH[m][0], wHy = P.WH[m][1], wHz = P.WH[m][2];
            const float cy = P.coef_e[1], cz = P.coef_e[2], cx = P.coef_e[0];
            if (comp == 0) {
                if (!pby && (rj == yl || rj == yh) && rk >= zl + pbz && rk <= zh && ri >= xl && ri <= xh - 1 + pbx) {
                    if (rj == yl) e = e - cy * d_inc(P, m, wHz, (float)ri + 0.5f, (float)yl - 0.5f, (float)rk, cntE) * P.wall_lo[1];
                    else e = e + cy * d_inc(P, m, wHz, (float)ri + 0.5f, (float)yh + 0.5f, (float)rk, cntE) * P.wall_hi[1];
                }
                if (!pbz && (rk == zl || rk == zh) && rj >= yl + pby && rj <= yh && ri >= xl && ri <= xh - 1 + pbx) {
                    if (rk == zl) e = e + cz * d_inc(P, m, wHy, (float)ri + 0.5f, (float)rj, (float)zl - 0.5f, cntE) * P.wall_lo[2];
                    else e = e - cz * d_inc(P, m, wHy, (float)ri + 0.5f, (float)rj, (float)zh + 0.5f, cntE) * P.wall_hi[2];
                }
            } else if (comp == 1) {
                if (!pbz && (rk == zl || rk == zh) && rj >= yl && rj <= yh - 1 + pby && ri >= xl + pbx && ri <= xh) {
                    if (rk == zl) e = e - cz * d_inc(P, m, wHx, (float)ri, (float)rj + 0.5f, (float)zl - 0.5f, cntE) * P.wall_lo[2];
                    else e = e + cz * d_inc(P, m, wHx, (float)ri, (float)rj + 0.5f, (float)zh + 0.5f, cntE) * P.wall_hi[2];
                }
                if (!pbx && (ri == xl || ri == xh) && rk >= zl + pbz && rk <= zh && rj >= yl && rj <= yh - 1 + pby) {
                    if (ri == xl) e = e + cx * d_inc(P, m, wHz, (float)xl - 0.5f, (float)rj + 0.5f, (float)rk, cntE) * P.wall_lo[0];
                    else e = e - cx * d_inc(P, m, wHz, (float)xh + 0.5f, (float)rj + 0.5f, (float)rk, cntE) * P.wall_hi[0];
                }
            } else {
                if (!pby && (rj == yl || rj == yh) && rk >= zl && rk <= zh - 1 + pbz && ri >= xl + pbx && ri <= xh) {
                    if (rj == yl) e = e + cy * d_inc(P, m, wHx, (float)ri, (float)yl - 0.5f, (float)rk + 0.5f, cntE) * P.wall_lo[1];
                    else e = e - cy * d_inc(P, m, wHx, (float)ri, (float)yh + 0.5f, (float)rk + 0.5f, cntE) * P.wall_hi[1];
                }
                if (!pbx && (ri == xl || ri == xh) && rk >= zl && rk <= zh - 1 + pbz && rj >= yl + pby && rj <= yh) {
                    if (ri == xl) e = e - cx * d_inc(P, m, wHy, (float)xl - 0.5f, (float)rj, (float)rk + 0.5f, cntE) * P.wall_lo[0];
                    else e = e + cx * d_inc(P, m, wHy, (float)xh + 0.5f, (float)rj, (float)rk + 0.5f, cntE) * P.wall_hi[0];
                }
            }
        }
    }
}

// One thread per (x, y) column marching its z chunk.  The per-cell work
// every position shares (bulk curl, CPML psi terms, periodic wraps) is
// straight-line code with per-lane predicates, so lanes in a CPML slab or
// at a wrap do not split a warp into two code paths; the rare corrections
// (sheet planes, TF/SF faces, the constant-k source plane) sit behind one
// flag per position, made of a column test done once and a plane test
// done per plane.  E(k+1) stays in registers as the next plane's E(k).
// The complex instantiation runs at 3 CTAs per SM (no spills).
template <typename T, bool SHEETS, bool TFSF>
__global__ void __launch_bounds__(256, sizeof(T) == sizeof(float) ? 5 : 3) k_update_h(const __grid_constant__ AemParams P, int counter) {
    counter = step_of(P, counter);
    const int NS = SHEETS ? P.nsheet : 0;  // decks without sheets compile the sheet code out
    const int px = blockIdx.x * 32 + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    // H is updated on reference indices 1..N-1 of every axis (all positions
    // of a periodic axis)
    const int hx = P.per[0] ? P.SX - 1 : P.SX - 2;
    const int hy = P.per[1] ? P.SY - 1 : P.SY - 2;
    const int hz = P.per[2] ? P.SZ - 1 : P.SZ - 2;
    __shared__ CoefTabs Tb;
    load_coef_tabs(P, Tb);
    if (px > hx || py > hy) return;
    const void *Ex = P.E[0], *Ey = P.E[1], *Ez = P.E[2];
    void *Hx = P.H[0], *Hy = P.H[1], *Hz = P.H[2];
    bool wx, wy;
    const int pxn = wrap_up(P, 0, px, P.SX, &wx);
    const int pyn = wrap_up(P, 1, py, P.SY, &wy);
    const long long plane = (long long)P.SY * P.PX;
    const long long offx = pxn - px, offy = (long long)(pyn - py) * P.PX;  // +x / +y neighbours
    const int i = px + 1, j = py + 1;
    const float DB = P.DB;
    const float dhx = P.den_h[0][i - 1], dhy = P.den_h[1][j - 1];
    const float cntH = (float)counter - 1.0f;
    // this column's CPML membership along x and y
    const int qx_lo = (i <= P.npml[0][0] - 1) ? i : 0;
    const int qx_hi = (i >= P.X + 1 - P.npml[0][1]) ? P.X - i : 0;
    const int qy_lo = (j <= P.npml[1][0] - 1) ? j : 0;
    const int qy_hi = (j >= P.Y + 1 - P.npml[1][1]) ? P.Y - j : 0;
    const bool col_cpml = qx_lo || qx_hi || qy_lo || qy_hi;
    // rare corrections that this column can take: an x or y sheet plane
    // through it, a TF/SF x or y face, the constant-k source plane
    bool col_rare = false;
    for (int s = 0; s < NS; s++)
        col_rare |= (P.sheet[s].axis == 0 && px == P.sheet[s].pos) || (P.sheet[s].axis == 1 && py == P.sheet[s].pos);
    if (TFSF && P.tfsf_on)
        col_rare |= (!P.per[0] && (i == P.lo[0] - 1 || i == P.hi[0])) || (!P.per[1] && (j == P.lo[1] - 1 || j == P.hi[1]));
    if (sizeof(T) != sizeof(float) && P.kmax_mode_TE)
        col_rare |= (P.kmax_src_axis == 0 && i == P.k_pl_H) || (P.kmax_src_axis == 1 && j == P.k_pl_H);

    // this CTA's z chunk
    const int pz0 = blockIdx.z * P.zch_h;
    const int pz_end = min(hz, ((int)blockIdx.z + 1) * P.zch_h - 1);
    long long c = lin(P, px, py, pz0);
    T ex = zero<T>(), ey = zero<T>();
    bool have = false;  // ex, ey of this plane were loaded as the previous plane's +z neighbours
    for (int pz = pz0; pz <= pz_end; pz++, c += plane) {
        bool wz;
        const int pzn = wrap_up(P, 2, pz, P.SZ, &wz);
        const long long offz = (long long)(pzn - pz) * plane;
        const int k = pz + 1;
        const float dhz = P.den_h[2][k - 1];
        if (!have) {
            ex = ld<T>(Ex, c);
            ey = ld<T>(Ey, c);
        }
        const T ez = ld<T>(Ez, c);
        const T ex_jp = ld_up<T>(P, Ex, c + offy, wy, 1);
        const T ex_kp = ld_up<T>(P, Ex, c + offz, wz, 2);
        const T ey_ip = ld_up<T>(P, Ey, c + offx, wx, 0);
        const T ey_kp = ld_up<T>(P, Ey, c + offz, wz, 2);
        const T ez_ip = ld_up<T>(P, Ez, c + offx, wx, 0);
        const T ez_jp = ld_up<T>(P, Ez, c + offy, wy, 1);
        bool rare = col_rare;
        for (int s = 0; s < NS; s++) rare |= P.sheet[s].axis == 2 && pz == P.sheet[s].pos;
        if (TFSF && P.tfsf_on) rare |= !P.per[2] && (k == P.lo[2] - 1 || k == P.hi[2]);
        if (sizeof(T) != sizeof(float) && P.kmax_mode_TE) rare |= P.kmax_src_axis == 2 && k == P.k_pl_H;

        T hxv = ld<T>(Hx, c), hyv = ld<T>(Hy, c), hzv = ld<T>(Hz, c);
        if (P.cpml_split != 2) {
        // bulk, ref :4448-4479 (DA = 1)
        hxv = hxv + DB * ((ez - ez_jp) * dhy + (ey_kp - ey) * dhz);
        hyv = hyv + DB * ((ez_ip - ez) * dhx + (ex - ex_kp) * dhz);
        hzv = hzv + DB * ((ey - ey_ip) * dhx + (ex_jp - ex) * dhy);

        if (rare) {
        // Smith-Maloney sheets, ref :4486-4554
        for (int s = 0; s < NS; s++) {
            const AemSheetPlane& S = P.sheet[s];
            const int pn = S.axis == 0 ? px : S.axis == 1 ? py : pz;
            if (pn != S.pos) continue;  // S.pos is a storage position
            const float f = DB * (P.sheet_thick / P.del[S.axis]);
            if (S.axis == 0) {
                const long long q = (long long)pz * S.pa + py;
                if (!S.nmask[q]) continue;
                const T es = ld<T>(S.es, q);
                const T es_kp = ld_up<T>(P, S.es, (long long)pzn * S.pa + py, wz, 2);
                const T es_jp = ld_up<T>(P, S.es, (long long)pz * S.pa + pyn, wy, 1);
                hyv = hyv + f * ((ex_kp - ex + es - es_kp) * dhz);
                hzv = hzv + f * ((ex - ex_jp + es_jp - es) * dhy);
            } else if (S.axis == 1) {
                const long long q = (long long)pz * S.pa + px;
                if (!S.nmask[q]) continue;
                const T es = ld<T>(S.es, q);
                const T es_kp = ld_up<T>(P, S.es, (long long)pzn * S.pa + px, wz, 2);
                const T es_ip = ld_up<T>(P, S.es, (long long)pz * S.pa + pxn, wx, 0);
                hxv = hxv + f * (ey - ey_kp + es_kp - es) * dhz;
                hzv = hzv + f * ((ey_ip - ey - es_ip + es) * dhx);
            } else {
                const long long q = (long long)py * S.pa + px;
                if (!S.nmask[q]) continue;
                const T es = ld<T>(S.es, q);
                const T es_jp = ld_up<T>(P, S.es, (long long)pyn * S.pa + px, wy, 1);
                const T es_ip = ld_up<T>(P, S.es, (long long)py * S.pa + pxn, wx, 0);
                hxv = hxv + f * (ez_jp - ez - es_jp + es) * dhy;
                hyv = hyv + f * ((ez - ez_ip + es_ip - es) * dhx);
            }
        }

        // incident fields on H
        if constexpr (sizeof(T) == sizeof(float)) {
            if constexpr (TFSF) tfsf_h(P, i, j, k, cntH, hxv, hyv, hzv);
        } else {
            if (P.kmax_mode_TE) {  // kmax TE plane on H, ref :4562-4624
                const int a = P.kmax_src_axis;
                const int ia = a == 0 ? i : a == 1 ? j : k;
                if (ia == P.k_pl_H) {
                    const float cf_ = P.coef_h[a];
                    const int lo0 = P.lo[0], hi0 = P.hi[0], lo1 = P.lo[1], hi1 = P.hi[1], lo2 = P.lo[2], hi2 = P.hi[2];
                    const float* kc = P.kcnt;
                    const float* kn = P.knum;
                    if (a == 0 && k >= lo2 && k <= hi2 && j >= lo1 && j <= hi1) {
                        hzv = hzv + cf_ * d_inc_k(P, P.WE[0][1], 0.0f, kc[1], ((float)j + 0.5f) * P.del[1], kc[2], (float)k * P.del[2], cntH, P.del[0]) * kn[2];
                        hyv = hyv + cf_ * d_inc_k(P, P.WE[0][2], 0.0f, kc[1], (float)j * P.del[1], kc[2], ((float)k + 0.5f) * P.del[2], cntH, P.del[0]) * kn[1];
                    }
                    if (a == 1 && k >= lo2 && k <= hi2 && i >= lo0 && i <= hi0) {
                        hzv = hzv + cf_ * d_inc_k(P, P.WE[0][0], 0.0f, kc[0], ((float)i + 0.5f) * P.del[0], kc[2], (float)k * P.del[2], cntH, P.del[1]) * kn[2];
                        hxv = hxv + cf_ * d_inc_k(P, P.WE[0][2], 0.0f, kc[0], (float)i * P.del[0], kc[2], ((float)k + 0.5f) * P.del[2], cntH, P.del[1]) * kn[0];
                    }
                    if (a == 2 && j >= lo1 && j <= hi1 && i >= lo0 && i <= hi0) {
                        hxv = hxv + cf_ * d_inc_k(P, P.WE[0][1], 0.0f, kc[1], ((float)j + 0.5f) * P.del[1], kc[0], (float)i * P.del[0], cntH, P.del[2]) * kn[0];
                        hyv = hyv + cf_ * d_inc_k(P, P.WE[0][0], 0.0f, kc[1], (float)j * P.del[1], kc[0], ((float)i + 0.5f) * P.del[0], cntH, P.del[2]) * kn[1];
                    }
                }
            }
        }
        }  // rare

        }  // cpml_split != 2
        // CPML on H, ref :5227-5375: Hx (y then z), Hy (x then z), Hz (x then y)
        const int qz_lo = (k <= P.npml[2][0] - 1) ? k : 0;
        const int qz_hi = (k >= P.Z + 1 - P.npml[2][1]) ? P.Z - k : 0;
        if (P.cpml_split != 1 && (col_cpml || qz_lo || qz_hi)) {
            if (qy_lo) hxv = hxv + DB * cpml_term<T>(P, P.psi_h[0][1][0], Tb.bh[1][0][qy_lo - 1], Tb.ch[1][0][qy_lo - 1], ez - ez_jp, P.del[1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]));
            if (qy_hi) hxv = hxv + DB * cpml_term<T>(P, P.psi_h[0][1][1], Tb.bh[1][1][qy_hi - 1], Tb.ch[1][1][qy_hi - 1], ez - ez_jp, P.del[1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]));
            if (qz_lo) hxv = hxv + DB * cpml_term<T>(P, P.psi_h[0][2][0], Tb.bh[2][0][qz_lo - 1], Tb.ch[2][0][qz_lo - 1], ey_kp - ey, P.del[2], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]));
            if (qz_hi) hxv = hxv + DB * cpml_term<T>(P, P.psi_h[0][2][1], Tb.bh[2][1][qz_hi - 1], Tb.ch[2][1][qz_hi - 1], ey_kp - ey, P.del[2], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]));
            if (qx_lo) hyv = hyv + DB * cpml_term<T>(P, P.psi_h[1][0][0], Tb.bh[0][0][qx_lo - 1], Tb.ch[0][0][qx_lo - 1], ez_ip - ez, P.del[0], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]));
            if (qx_hi) hyv = hyv + DB * cpml_term<T>(P, P.psi_h[1][0][1], Tb.bh[0][1][qx_hi - 1], Tb.ch[0][1][qx_hi - 1], ez_ip - ez, P.del[0], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]));
            if (qz_lo) hyv = hyv + DB * cpml_term<T>(P, P.psi_h[1][2][0], Tb.bh[2][0][qz_lo - 1], Tb.ch[2][0][qz_lo - 1], ex - ex_kp, P.del[2], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]));
            if (qz_hi) hyv = hyv + DB * cpml_term<T>(P, P.psi_h[1][2][1], Tb.bh[2][1][qz_hi - 1], Tb.ch[2][1][qz_hi - 1], ex - ex_kp, P.del[2], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]));
            if (qx_lo) hzv = hzv + DB * cpml_term<T>(P, P.psi_h[2][0][0], Tb.bh[0][0][qx_lo - 1], Tb.ch[0][0][qx_lo - 1], ey - ey_ip, P.del[0], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]));
            if (qx_hi) hzv = hzv + DB * cpml_term<T>(P, P.psi_h[2][0][1], Tb.bh[0][1][qx_hi - 1], Tb.ch[0][1][qx_hi - 1], ey - ey_ip, P.del[0], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]));
            if (qy_lo) hzv = hzv + DB * cpml_term<T>(P, P.psi_h[2][1][0], Tb.bh[1][0][qy_lo - 1], Tb.ch[1][0][qy_lo - 1], ex_jp - ex, P.del[1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]));
            if (qy_hi) hzv = hzv + DB * cpml_term<T>(P, P.psi_h[2][1][1], Tb.bh[1][1][qy_hi - 1], Tb.ch[1][1][qy_hi - 1], ex_jp - ex, P.del[1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]));
        }
        st<T>(Hx, c, hxv);
        st<T>(Hy, c, hyv);
        st<T>(Hz, c, hzv);
        // E(k+1) is the next plane's E(k) (not across a periodic wrap; FP32
        // only: the complex kernel keeps its registers for more CTAs)
        ex = ex_kp;
        ey = ey_kp;
        have = sizeof(T) == sizeof(float) && !wz;
    }
}

// Material coefficients of one E edge: sheet override, index-1 vacuum
// default, uniform-neighbourhood table or the reference's 4-cell average.
// The Drude coefficients of the edge are not kept here (they would live in
// local memory): drude_coef recomputes them from the ids inside the Drude box.
struct EdgeCoef {
    float ga, gb;
    int i0, i1, i2, i3;  // the four cell ids
    bool uni;            // the four ids are equal: table values
};

// Ja, Jb of pole p of an edge, ref :2859-2895 (4-cell average of wp, gamma)
__device__ inline void drude_coef(const AemParams& P, int c, const EdgeCoef& co, int p, float& ja, float& jb) {
    if (co.uni) {
        ja = P.ucoef[co.i0].ja[p][c];
        jb = P.ucoef[co.i0].jb[p][c];
        return;
    }
    const AemMaterial *m0 = P.mat + co.i0, *m1 = P.mat + co.i1, *m2 = P.mat + co.i2, *m3 = P.mat + co.i3;
    const float w = (m0->wp[p][c] + m1->wp[p][c] + m2->wp[p][c] + m3->wp[p][c]) / 4.0f;
    const float g = (m0->gam[p][c] + m1->gam[p][c] + m2->gam[p][c] + m3->gam[p][c]) / 4.0f;
    ja = d_ja(g, P.dt);
    jb = d_jb(w, g, P.dt);
}

// i0..i3: the ids of the four cells around the edge in the reference's
// order (ref :2516-2527), all 0 on an unaveraged wall edge
__device__ inline void edge_coef(const AemParams& P, const CoefTabs& Tb, int c, int i0, int i1, int i2, int i3,
                                 EdgeCoef& o) {
    o.i0 = i0; o.i1 = i1; o.i2 = i2; o.i3 = i3;
    o.uni = o.i0 == o.i1 && o.i0 == o.i2 && o.i0 == o.i3;
    if (o.uni) {
        o.ga = Tb.ga[o.i0][c];
        o.gb = Tb.gb[o.i0][c];
        return;
    }
    const float e = (Tb.eps[o.i0][c] + Tb.eps[o.i1][c] + Tb.eps[o.i2][c] + Tb.eps[o.i3][c]) / 4.0f;
    const float s = (Tb.sig[o.i0][c] + Tb.sig[o.i1][c] + Tb.sig[o.i2][c] + Tb.sig[o.i3][c]) / 4.0f;
    float tp = 0.0f;
    for (int p = 0; p < P.npoles; p++) {
        float ja, jb;
        drude_coef(P, c, o, p, ja, jb);
        tp = tp + jb;
    }
    o.ga = d_ga(s + tp, e, P.dt);
    o.gb = d_gb(s + tp, e, P.dt);
}

// sheet-plane Ga/Gb override of E component c at this position, if any
__device__ inline bool sheet_override(const AemParams& P, int c, int px, int py, int pz, float* ga, float* gb) {
    for (int s = 0; s < P.nsheet; s++) {
        const AemSheetPlane& S = P.sheet[s];
        if (S.axis == c) continue;
        const int pn = S.axis == 0 ? px : S.axis == 1 ? py : pz;
        if (pn != S.pos) continue;
        const int ua = S.axis == 0 ? 1 : 0;
        const int pa = ua == 0 ? px : py;
        const int pb = S.axis == 2 ? py : pz;
        const long long q = (long long)pb * S.pa + pa;
        const int bit = c == ua ? 1 : 2;
        if (!(S.tmask[q] & bit)) continue;
        *ga = bit == 1 ? S.ga1[q] : S.ga2[q];
        *gb = bit == 1 ? S.gb1[q] : S.gb2[q];
        return true;
    }
    return false;
}

// Drude ADE of one E edge inside its bounding box, ref :5794-5802
template <typename T>
__device__ inline T drude_update(const AemParams& P, int c, int px, int py, int pz, T e_new, T e_old, float gb,
                                 const EdgeCoef& co) {
    const int ox = P.jorg[c][0], oy = P.jorg[c][1], oz = P.jorg[c][2];
    const int nx = P.jext[c][0], ny = P.jext[c][1], nz = P.jext[c][2];
    const int lx = px - ox, ly = py - oy, lz = pz - oz;
    if (lx < 0 || ly < 0 || lz < 0 || lx >= nx || ly >= ny || lz >= nz) return e_new;
    void* J = P.jsrc[c];
    const long long vol = (long long)nx * ny * nz, base = ((long long)lz * ny + ly) * nx + lx;
    T t = zero<T>();
    for (int p = 0; p < P.npoles; p++) {
        float ja, jb;
        drude_coef(P, c, co, p, ja, jb);
        t = t + (1.0f + ja) * ld<T>(J, p * vol + base);
    }
    const T e = e_new - gb * t / 2.0f;
    for (int p = 0; p < P.npoles; p++) {
        float ja, jb;
        drude_coef(P, c, co, p, ja, jb);
        st<T>(J, p * vol + base, ja * ld<T>(J, p * vol + base) + jb * (e + e_old));
    }
    return e;
}

__device__ inline bool in_box(const AemParams& P, int c, int ri, int rj, int rk) {
    const int* b = P.dbox[c];
    return rk >= b[0] && rk <= b[1] && rj >= b[2] && rj <= b[3] && ri >= b[4] && ri <= b[5];
}

// DRUDE: the instantiation for decks with Drude poles.  Same structure as
// k_update_h: CPML, walls and wraps are per-lane work on the common path,
// sheets, Drude boxes, TF/SF faces and the constant-k source plane sit
// behind one flag per position, and H(k-1) and the ids of plane k-1 come
// from the previous plane (FP32; the complex kernel reloads them and runs
// 3 CTAs per SM without Drude poles, which overlaps better in a batch of
// constant-k runs: 0.79 s against 1.00 s at 2 CTAs for 64 unit cells).
template <typename T, bool DRUDE, bool SHEETS, bool TFSF>
__global__ void __launch_bounds__(256, sizeof(T) == sizeof(float) ? 3 : (DRUDE ? 2 : 3)) k_update_e(const __grid_constant__ AemParams P, int counter) {
    counter = step_of(P, counter);
    const int NS = SHEETS ? P.nsheet : 0;  // decks without sheets compile the sheet code out
    const int px = blockIdx.x * 32 + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    __shared__ CoefTabs Tb;
    load_coef_tabs(P, Tb);
    if (px >= P.SX || py >= P.SY) return;
    const void *Hx = P.H[0], *Hy = P.H[1], *Hz = P.H[2];
    void *Ex = P.E[0], *Ey = P.E[1], *Ez = P.E[2];
    // update ranges, ref :5670-5702: the normal component covers reference
    // indices 1..N-1 of its own axis, tangential axes 2..N-1 (walls stay 0)
    auto upd = [&](int a, int p, bool normal) {
        const int S = a == 0 ? P.SX : a == 1 ? P.SY : P.SZ;
        if (P.per[a]) return true;
        return normal ? (p <= S - 2) : (p >= 1 && p <= S - 2);
    };
    const bool ex_xy = upd(0, px, true) && upd(1, py, false);
    const bool ey_xy = upd(0, px, false) && upd(1, py, true);
    const bool ez_xy = upd(0, px, false) && upd(1, py, false);
    if (!ex_xy && !ey_xy && !ez_xy) return;
    bool wxd, wyd;
    int pxd = wrap_dn(P, 0, px, P.SX, &wxd);
    int pyd = wrap_dn(P, 1, py, P.SY, &wyd);
    if (pxd < 0) pxd = 0;  // only read by components not updated here
    if (pyd < 0) pyd = 0;
    const int i = px + 1, j = py + 1;
    const float dex = P.den_e[0][i - 1], dey = P.den_e[1][j - 1];
    const float cntE = (float)counter - 0.5f;
    // representative reference indices for bound tests (periodic axes)
    const int rix_t = rep_idx(P, 0, px, true), riy_t = rep_idx(P, 1, py, true);
    const int qxl = (i >= 2 && i <= P.npml[0][0]) ? i : 0, qxh = (i >= P.X + 1 - P.npml[0][1] && i <= P.X - 1) ? P.X + 1 - i : 0;
    const int qyl = (j >= 2 && j <= P.npml[1][0]) ? j : 0, qyh = (j >= P.Y + 1 - P.npml[1][1] && j <= P.Y - 1) ? P.Y + 1 - j : 0;
    const bool x_unavg = !P.per[0] && i == 1, y_unavg = !P.per[1] && j == 1;
    const long long plane = (long long)P.SY * P.PX;
    const long long offx = pxd - px, offy = (long long)(pyd - py) * P.PX;  // -x / -y neighbours
    const bool col_cpml = qxl || qxh || qyl || qyh;
    // rare corrections that this column can take: an x or y sheet plane
    // through it, a TF/SF x or y face, the constant-k source plane, a
    // Drude box over it
    bool col_rare = false;
    for (int s = 0; s < NS; s++)
        col_rare |= (P.sheet[s].axis == 0 && px == P.sheet[s].pos) || (P.sheet[s].axis == 1 && py == P.sheet[s].pos);
    if (TFSF && P.tfsf_on)
        col_rare |= (!P.per[0] && (i == P.lo[0] || i == P.hi[0])) || (!P.per[1] && (j == P.lo[1] || j == P.hi[1]));
    if (sizeof(T) != sizeof(float) && P.kmax_mode_TM)
        col_rare |= (P.kmax_src_axis == 0 && (i == P.k_pl_E || rix_t == P.k_pl_E)) ||
                    (P.kmax_src_axis == 1 && (j == P.k_pl_E || riy_t == P.k_pl_E));
    bool col_drude = false;
    if (DRUDE && P.has_drude)
        for (int cc = 0; cc < 3; cc++) {
            const int* b = P.dbox[cc];
            const int ri = cc == 0 ? i : rix_t, rj = cc == 1 ? j : riy_t;
            col_drude |= rj >= b[2] && rj <= b[3] && ri >= b[4] && ri <= b[5];
        }

    const int pz0 = blockIdx.z * P.zch_e;
    const int pz_end = min(P.SZ, ((int)blockIdx.z + 1) * P.zch_e);
    long long c = lin(P, px, py, pz0);
    // H(k-1) and the ids of plane k-1 from the previous plane
    T hx_prev = zero<T>(), hy_prev = zero<T>();
    int id0_prev = 0, idx_prev = 0, idy_prev = 0;
    bool have = false;
    for (int pz = pz0; pz < pz_end; pz++, c += plane) {
        const bool ex_u = ex_xy && upd(2, pz, false), ey_u = ey_xy && upd(2, pz, false), ez_u = ez_xy && upd(2, pz, true);
        if (!ex_u && !ey_u && !ez_u) {
            have = false;
            continue;
        }
        bool wzd;
        int pzd = wrap_dn(P, 2, pz, P.SZ, &wzd);
        if (pzd < 0) pzd = 0;
        const long long offz = (long long)(pzd - pz) * plane;
        const bool reuse = have && !wzd;
        const int k = pz + 1;
        const int riz_t = rep_idx(P, 2, pz, true);
        const float dez = P.den_e[2][k - 1];
        const bool unavg = x_unavg || y_unavg || (!P.per[2] && k == 1);
        const int qzl = (k >= 2 && k <= P.npml[2][0]) ? k : 0, qzh = (k >= P.Z + 1 - P.npml[2][1] && k <= P.Z - 1) ? P.Z + 1 - k : 0;
        // Every global load of the plane is issued before any update, so a
        // thread waits on one round of memory latency instead of one per
        // component.  A neighbour index of a component not updated here is
        // clamped to 0 above and its value is not used.
        const T hx = ld<T>(Hx, c), hy = ld<T>(Hy, c), hz = ld<T>(Hz, c);
        const T hz_jm = ld_dn<T>(P, Hz, c + offy, wyd, 1);
        const T hy_km = reuse ? hy_prev : ld_dn<T>(P, Hy, c + offz, wzd, 2);
        const T hz_im = ld_dn<T>(P, Hz, c + offx, wxd, 0);
        const T hx_km = reuse ? hx_prev : ld_dn<T>(P, Hx, c + offz, wzd, 2);
        const T hy_im = ld_dn<T>(P, Hy, c + offx, wxd, 0), hx_jm = ld_dn<T>(P, Hx, c + offy, wyd, 1);
        const T eo0 = ld<T>(Ex, c), eo1 = ld<T>(Ey, c), eo2 = ld<T>(Ez, c);
        // the seven cells around this position's three edges, ref :2516-2527
        int id0 = 0, idx = 0, idy = 0, idz = 0, idxy = 0, idxz = 0, idyz = 0;
        if (!unavg) {
            const uint8_t* C = P.cell;
            id0 = C[c]; idx = C[c + offx]; idy = C[c + offy]; idxy = C[c + offx + offy];
            if (reuse) {
                idz = id0_prev; idxz = idx_prev; idyz = idy_prev;
            } else {
                idz = C[c + offz]; idxz = C[c + offx + offz]; idyz = C[c + offy + offz];
            }
        }
        hx_prev = hx;
        hy_prev = hy;
        id0_prev = id0;
        idx_prev = idx;
        idy_prev = idy;
        have = sizeof(T) == sizeof(float) && !unavg;  // the ids of this plane were read (FP32 only, as in H)
        bool rare = col_rare;
        for (int s = 0; s < NS; s++) rare |= P.sheet[s].axis == 2 && pz == P.sheet[s].pos;
        if (TFSF && P.tfsf_on) rare |= !P.per[2] && (k == P.lo[2] || k == P.hi[2]);
        if (sizeof(T) != sizeof(float) && P.kmax_mode_TM)
            rare |= P.kmax_src_axis == 2 && (k == P.k_pl_E || riz_t == P.k_pl_E);
        if (col_drude)
            for (int cc = 0; cc < 3; cc++) {
                const int rk = cc == 2 ? k : riz_t;
                rare |= rk >= P.dbox[cc][0] && rk <= P.dbox[cc][1];
            }
        const bool cpml_here = col_cpml || qzl || qzh;
        // a sheet plane through this position (both sheet loops below act
        // only there)
        bool sheet_here = false;
        for (int s = 0; s < NS; s++) {
            const AemSheetPlane& S = P.sheet[s];
            sheet_here |= (S.axis == 0 ? px : S.axis == 1 ? py : pz) == S.pos;
        }

#pragma unroll
        for (int comp = 0; comp < 3; comp++) {
            if ((comp == 0 && !ex_u) || (comp == 1 && !ey_u) || (comp == 2 && !ez_u)) continue;
            void* Ec = P.E[comp];
            // curl of H, ref :5673-5705
            T d1, d2;   // the two difference terms (second minus first neighbour as in the reference)
            float den1, den2;
            EdgeCoef co;
            if (comp == 0) {
                d1 = hz - hz_jm; den1 = dey; d2 = hy_km - hy; den2 = dez;
                edge_coef(P, Tb, 0, id0, idy, idz, idyz, co);
            } else if (comp == 1) {
                d1 = hz_im - hz; den1 = dex; d2 = hx - hx_km; den2 = dez;
                edge_coef(P, Tb, 1, id0, idx, idz, idxz, co);
            } else {
                d1 = hy - hy_im; den1 = dex; d2 = hx_jm - hx; den2 = dey;
                edge_coef(P, Tb, 2, id0, idx, idy, idxy, co);
            }
            const T curl = d1 * den1 + d2 * den2;
            float ga = co.ga, gb = co.gb;
            if (sheet_here) sheet_override(P, comp, px, py, pz, &ga, &gb);
            const T eold = comp == 0 ? eo0 : comp == 1 ? eo1 : eo2;
            T e = eold;
            if (P.cpml_split != 2) {
            e = ga * eold + gb * curl;

            // sheet sub-cell field of the normal component, ref :5714-5780
            for (int s = 0; sheet_here && s < NS; s++) {
                const AemSheetPlane& S = P.sheet[s];
                if (S.axis != comp) continue;
                const int pn = comp == 0 ? px : comp == 1 ? py : pz;
                if (pn != S.pos) continue;
                const int pa = comp == 0 ? py : px, pb = comp == 2 ? py : pz;
                const long long q = (long long)pb * S.pa + pa;
                if (!S.nmask[q]) continue;
                st<T>(S.es, q, S.sa[q] * ld<T>(S.es, q) + S.sb[q] * curl);
            }
            if (rare) {
            // representative indices of this component
            const int ri = comp == 0 ? px + 1 : rix_t, rj = comp == 1 ? py + 1 : riy_t, rk = comp == 2 ? pz + 1 : riz_t;
            if (DRUDE && P.has_drude && in_box(P, comp, ri, rj, rk)) e = drude_update<T>(P, comp, px, py, pz, e, eold, gb, co);

            if constexpr (sizeof(T) == sizeof(float)) {
                if constexpr (TFSF) tfsf_e(P, comp, ri, rj, rk, cntE, e);
            } else {
                if (P.kmax_mode_TM) {  // kmax TM plane on E, ref :5861-5947
                    const int a = P.kmax_src_axis;
                    const int ia = a == 0 ? ri : a == 1 ? rj : rk;
                    if (ia == P.k_pl_E) {
                        const float cf_ = P.coef_e[a];
                        const float* kc = P.kcnt;
                        const float* kn = P.knum;
                        const float fi = (float)(px + 1), fj = (float)(py + 1), fk = (float)(pz + 1);
                        const float dx = P.del[0], dy = P.del[1], dz = P.del[2];
                        if (a == 0) {
                            if (comp == 2 && rk >= 1 && rk <= P.Z - 1 && rj >= 2 && rj <= P.Y - 1)
                                e = e + cf_ * d_inc_k(P, P.WH[0][1], -0.5f, kc[1], fj * dy, kc[2], (fk + 0.5f) * dz, cntE, dx) * kn[2];
                            if (comp == 1 && rk >= 2 && rk <= P.Z - 1 && rj >= 1 && rj <= P.Y - 1)
                                e = e + cf_ * d_inc_k(P, P.WH[0][2], -0.5f, kc[1], (fj + 0.5f) * dy, kc[2], fk * dz, cntE, dx) * kn[1];
                        } else if (a == 1) {
                            if (comp == 2 && rk >= 1 && rk <= P.Z - 1 && ri >= 2 && ri <= P.X - 1)
                                e = e + cf_ * d_inc_k(P, P.WH[0][0], -0.5f, kc[0], fi * dx, kc[2], (fk + 0.5f) * dz, cntE, dy) * kn[2];
                            if (comp == 0 && rk >= 2 && rk <= P.Z - 1 && ri >= 1 && ri <= P.X - 1)
                                e = e + cf_ * d_inc_k(P, P.WH[0][2], -0.5f, kc[0], (fi + 0.5f) * dx, kc[2], fk * dz, cntE, dy) * kn[0];
                        } else {
                            if (comp == 0 && rj >= 2 && rj <= P.Y - 1 && ri >= 1 && ri <= P.X - 1)
                                e = e + cf_ * d_inc_k(P, P.WH[0][1], -0.5f, kc[1], fj * dy, kc[0], (fi + 0.5f) * dx, cntE, dz) * kn[0];
                            if (comp == 1 && rj >= 1 && rj <= P.Y - 1 && ri >= 2 && ri <= P.X - 1)
                                e = e + cf_ * d_inc_k(P, P.WH[0][0], -0.5f, kc[1], (fj + 0.5f) * dy, kc[0], fi * dx, cntE, dz) * kn[1];
                        }
                    }
                }
            }
            }  // rare

            }  // cpml_split != 2
            // CPML on E, ref :6522-6670: Ex (y then z), Ey (x then z), Ez (x then y)
            if (P.cpml_split == 1 || !cpml_here) {
                st<T>(Ec, c, e);
                continue;
            }
            const int ax1 = comp == 0 ? 1 : 0, ax2 = comp == 2 ? 1 : 2;
            const int q1l = ax1 == 0 ? qxl : qyl, q1h = ax1 == 0 ? qxh : qyh;
            const int q2l = ax2 == 1 ? qyl : qzl, q2h = ax2 == 1 ? qyh : qzh;
            const T t1 = comp == 2 ? d1 : (comp == 0 ? d1 : d1);  // difference along ax1
            const T t2 = d2;                                     // difference along ax2
            if (q1l) e = e + gb * cpml_term<T>(P, P.psi_e[comp][ax1][0], Tb.be[ax1][0][q1l - 1], Tb.ce[ax1][0][q1l - 1], t1, P.del[ax1], psi_idx(P, ax1, q1l, px, py, pz, P.npml[ax1][0]));
            if (q1h) e = e + gb * cpml_term<T>(P, P.psi_e[comp][ax1][1], Tb.be[ax1][1][q1h - 1], Tb.ce[ax1][1][q1h - 1], t1, P.del[ax1], psi_idx(P, ax1, q1h, px, py, pz, P.npml[ax1][1]));
            if (q2l) e = e + gb * cpml_term<T>(P, P.psi_e[comp][ax2][0], Tb.be[ax2][0][q2l - 1], Tb.ce[ax2][0][q2l - 1], t2, P.del[ax2], psi_idx(P, ax2, q2l, px, py, pz, P.npml[ax2][0]));
            if (q2h) e = e + gb * cpml_term<T>(P, P.psi_e[comp][ax2][1], Tb.be[ax2][1][q2h - 1], Tb.ce[ax2][1][q2h - 1], t2, P.del[ax2], psi_idx(P, ax2, q2h, px, py, pz, P.npml[ax2][1]));
            st<T>(Ec, c, e);
        }
    }
}

// ---------------------------------------------------------------------------
// TF/SF corrections in their own kernels (FP32 runs whose TF/SF faces stay
// clear of every CPML slab, P.tfsf_sep): the shell of the TF/SF box, each
// position once, after the bulk pass of its field.  The reference applies
// them after the bulk, sheet and Drude terms and before the CPML terms; no
// CPML term reaches these positions, so adding them afterwards is the same
// sequence of operations.  Per axis a the shell spans reference indices
// r0..r1 (the whole axis when periodic) and its faces sit at f0, f1 (none
// when periodic); group X takes the x faces, Y the y faces off them, Z the
// rest.
struct Shell {
    int r0[3], n[3], f[3][2], nf[3];
};
__device__ inline bool shell_cell(const Shell& S, long long t, int idx[3]) {
    const int nx = S.n[0], ny = S.n[1], nz = S.n[2];
    const int mx = nx - S.nf[0], my = ny - S.nf[1];  // x / y positions off the faces
    auto off = [&](int a, int q) {                    // q-th index of axis a that is not a face
        int v = S.r0[a] + q;
        for (int u = 0; u < S.nf[a]; u++)
            if (v >= S.f[a][u]) v++;
        return v;
    };
    long long gx = (long long)S.nf[0] * ny * nz, gy = (long long)S.nf[1] * mx * nz, gz = (long long)S.nf[2] * mx * my;
    if (t < gx) {
        idx[0] = S.f[0][t / ((long long)ny * nz)];
        const long long r = t % ((long long)ny * nz);
        idx[1] = S.r0[1] + (int)(r % ny);
        idx[2] = S.r0[2] + (int)(r / ny);
        return true;
    }
    t -= gx;
    if (t < gy) {
        idx[1] = S.f[1][t / ((long long)mx * nz)];
        const long long r = t % ((long long)mx * nz);
        idx[0] = off(0, (int)(r % mx));
        idx[2] = S.r0[2] + (int)(r / mx);
        return true;
    }
    t -= gy;
    if (t < gz) {
        idx[2] = S.f[2][t / ((long long)mx * my)];
        const long long r = t % ((long long)mx * my);
        idx[0] = off(0, (int)(r % mx));
        idx[1] = off(1, (int)(r / mx));
        return true;
    }
    return false;
}

__global__ void k_tfsf_h(const __grid_constant__ AemParams P, const Shell S, long long total, int counter) {
    counter = step_of(P, counter);
    const float cntH = (float)counter - 1.0f;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int idx[3];
        if (!shell_cell(S, t, idx)) continue;
        const long long c = lin(P, idx[0] - 1, idx[1] - 1, idx[2] - 1);
        float* Hx = reinterpret_cast<float*>(P.H[0]);
        float* Hy = reinterpret_cast<float*>(P.H[1]);
        float* Hz = reinterpret_cast<float*>(P.H[2]);
        float hx = Hx[c], hy = Hy[c], hz = Hz[c];
        tfsf_h(P, idx[0], idx[1], idx[2], cntH, hx, hy, hz);
        Hx[c] = hx;
        Hy[c] = hy;
        Hz[c] = hz;
    }
}

__global__ void k_tfsf_e(const __grid_constant__ AemParams P, const Shell S, long long total, int counter) {
    counter = step_of(P, counter);
    const float cntE = (float)counter - 0.5f;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int idx[3];
        if (!shell_cell(S, t, idx)) continue;
        const int px = idx[0] - 1, py = idx[1] - 1, pz = idx[2] - 1;
        // the components k_update_e updates here (ref :5670-5702)
        auto upd = [&](int a, int p, bool normal) {
            const int Sa = a == 0 ? P.SX : a == 1 ? P.SY : P.SZ;
            if (P.per[a]) return true;
            return normal ? (p <= Sa - 2) : (p >= 1 && p <= Sa - 2);
        };
        const bool u[3] = {upd(0, px, true) && upd(1, py, false) && upd(2, pz, false),
                           upd(0, px, false) && upd(1, py, true) && upd(2, pz, false),
                           upd(0, px, false) && upd(1, py, false) && upd(2, pz, true)};
        const int rix_t = rep_idx(P, 0, px, true), riy_t = rep_idx(P, 1, py, true), riz_t = rep_idx(P, 2, pz, true);
        const long long c = lin(P, px, py, pz);
        for (int comp = 0; comp < 3; comp++) {
            if (!u[comp]) continue;
            float* Ec = reinterpret_cast<float*>(P.E[comp]);
            float e = Ec[c];
            const int ri = comp == 0 ? px + 1 : rix_t, rj = comp == 1 ? py + 1 : riy_t, rk = comp == 2 ? pz + 1 : riz_t;
            tfsf_e(P, comp, ri, rj, rk, cntE, e);
            Ec[c] = e;
        }
    }
}

// the shell of H (faces lo-1, hi) or E (faces lo, hi)
static long long tfsf_shell(const AemParams& P, bool e, Shell& S) {
    const int Sx[3] = {P.SX, P.SY, P.SZ};
    long long cells = 1;
    for (int a = 0; a < 3; a++) {
        if (P.per[a]) {
            S.r0[a] = 1;
            S.n[a] = Sx[a];
            S.nf[a] = 0;
        } else {
            const int f0 = e ? P.lo[a] : P.lo[a] - 1, f1 = P.hi[a];
            S.r0[a] = f0;
            S.n[a] = f1 - f0 + 1;
            S.f[a][0] = f0;
            S.f[a][1] = f1;
            S.nf[a] = f1 > f0 ? 2 : 1;
        }
        if (S.n[a] <= 0) return 0;
        cells *= S.n[a];
    }
    const long long mx = S.n[0] - S.nf[0], my = S.n[1] - S.nf[1];
    return (long long)S.nf[0] * S.n[1] * S.n[2] + (long long)S.nf[1] * mx * S.n[2] + (long long)S.nf[2] * mx * my;
}

static int launch_tfsf(const AemParams& P, bool e, int counter, cudaStream_t s) {
    Shell S{};
    const long long total = tfsf_shell(P, e, S);
    if (total <= 0) return 0;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 8);
    if (e) k_tfsf_e<<<blocks, 256, 0, s>>>(P, S, total, counter);
    else k_tfsf_h<<<blocks, 256, 0, s>>>(P, S, total, counter);
    return 1;
}

// ---------------------------------------------------------------------------
// a launch shape the caller did not set takes the default
static void upd_shape(int& zch, int& ty) {
    if (zch < 1) zch = UPD_ZCH;
    if (ty < 1 || ty > 8) ty = UPD_TY;
}

int launch_update_h(const AemParams& Pin, int counter, cudaStream_t s) {
    AemParams P = Pin;
    upd_shape(P.zch_h, P.ty_h);
    dim3 blk(32, P.ty_h), grd((P.SX + 31) / 32, (P.SY + P.ty_h - 1) / P.ty_h, (P.SZ + P.zch_h - 1) / P.zch_h);
    const bool sh = P.nsheet > 0;
    // TF/SF inside the update kernel unless its own kernel applies it
    const bool tf = P.tfsf_on && !P.tfsf_sep;
    if (P.kmax) {
        if (sh) k_update_h<cf, true, false><<<grd, blk, 0, s>>>(P, counter);
        else k_update_h<cf, false, false><<<grd, blk, 0, s>>>(P, counter);
    } else if (tf) {
        if (sh) k_update_h<float, true, true><<<grd, blk, 0, s>>>(P, counter);
        else k_update_h<float, false, true><<<grd, blk, 0, s>>>(P, counter);
    } else {
        if (sh) k_update_h<float, true, false><<<grd, blk, 0, s>>>(P, counter);
        else k_update_h<float, false, false><<<grd, blk, 0, s>>>(P, counter);
    }
    if (!P.kmax && P.tfsf_on && P.tfsf_sep && P.cpml_split != 2) return 1 + launch_tfsf(P, false, counter, s);
    return 1;
}
template <typename T, bool DRUDE, bool TFSF>
static void launch_e(const AemParams& P, int counter, dim3 grd, dim3 blk, cudaStream_t s) {
    if (P.nsheet > 0) k_update_e<T, DRUDE, true, TFSF><<<grd, blk, 0, s>>>(P, counter);
    else k_update_e<T, DRUDE, false, TFSF><<<grd, blk, 0, s>>>(P, counter);
}

int launch_update_e(const AemParams& Pin, int counter, cudaStream_t s) {
    AemParams P = Pin;
    upd_shape(P.zch_e, P.ty_e);
    dim3 blk(32, P.ty_e), grd((P.SX + 31) / 32, (P.SY + P.ty_e - 1) / P.ty_e, (P.SZ + P.zch_e - 1) / P.zch_e);
    if (P.kmax) {
        if (P.has_drude) launch_e<cf, true, false>(P, counter, grd, blk, s);
        else launch_e<cf, false, false>(P, counter, grd, blk, s);
    } else {
        const bool tf = P.tfsf_on && !P.tfsf_sep;
        if (P.has_drude) {
            if (tf) launch_e<float, true, true>(P, counter, grd, blk, s);
            else launch_e<float, true, false>(P, counter, grd, blk, s);
        } else {
            if (tf) launch_e<float, false, true>(P, counter, grd, blk, s);
            else launch_e<float, false, false>(P, counter, grd, blk, s);
        }
        if (P.tfsf_on && P.tfsf_sep && P.cpml_split != 2) return 1 + launch_tfsf(P, true, counter, s);
    }
    return 1;
}

}  // namespace aem
