// aem_design.cu -- the design-gradient engine (aem_design.h): forward and
// adjoint updates over FP32 or FP64 state, checkpointing and the gradient.
//
// Forward step n (reference order, fdtd_solver.f90:4440-8299, restricted to
// bulk Yee + CPML + lumped ports):
//   k_dsn_h        H bulk (:4442-4484) and CPML H (:5227-5375)
//   k_dsn_ports_h  loop current, line currents, current source (:4800-5011)
//   k_dsn_e        E bulk (:5667-5710) with design-box Ga/Gb, CPML E
//                  (:6522-6670); design-box E is recorded for the gradient
//   k_dsn_ports_e  line voltages, voltage source, port E (:6123-6283), and
//                  the probe DFT
// The FP32 instantiation evaluates every expression as the production
// kernels do (aem_kernels.cu, aem_aux.cu), so with the deck's own materials
// in the design box it reproduces the solver's fields bit for bit.
//
// Adjoint step n undoes forward step n transposed, last operation first:
//   k_adj_grad     gradient sums of step n (design edges)
//   k_adj_ports_e  probe DFT seed, port E / line voltages transposed
//   k_adj_h        E bulk + CPML E transposed, gathered onto H faces
//   k_adj_ports_h  line currents and loop current transposed
//   k_adj_e        H bulk + CPML H transposed, gathered onto E edges
// Notation: lE, lH are the adjoints of E^n, H^{n-1/2}.  The E-side state
// kept is w = Gb lE (lE itself is needed only on design and port edges, as
// w / Gb), so the adjoint moves as many bytes per step as the forward pass.
// se = the adjoint of the E psi value just written (b-scaled psi adjoint plus
// w), sh likewise for H (b sh_next + DB lH).  The CPML, port and probe
// edges never meet the design box or each other (checked on the host), which
// lets each transposed operation sit in the kernel that owns its cells.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "aem_design.h"
#include "aem_dev.cuh"
#include "aem_kernels.h"
#include "aem_solver.h"

#define DSN_CUDA(x)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_)); \
    } while (0)

namespace aem {
namespace {

constexpr int DZCH = 16;  // z planes per CTA of the volume kernels

template <typename R>
struct DsnDev {
    R* E[3];
    R* H[3];
    R* pe[3][3][2];  // CPML psi, [component][slab axis][side]
    R* ph[3][3][2];
    R* lH[3];
    R* w[3];
    R* se[3][3][2];
    R* sh[3][3][2];
    R* V[AEM_MAX_PORTS];
    R* I[AEM_MAX_PORTS];
    R* lV[AEM_MAX_PORTS];
    R* lI[AEM_MAX_PORTS];
    int lo[3], n[3];        // design cells, storage positions
    int eo[3][3], en[3][3];  // edge box of each component: origin, extents
    long long eoff[3], nedge;
    const R* eps;
    const R* sig;  // null: the cells' own conductivity
    R* ga;
    R* gb;
    R* rec;        // [slot][edge]
    double* A;     // sum lE^n E^{n-1}
    double* B;     // sum lE^n (E^n - Ga E^{n-1})
    int pc, ppx, ppy, ppz;
    long long pidx;
    double fdt2;   // 2 f dt
    double* dft;
    int acc_dft;
    double* ov;    // [edge][4]: DFTs at the probe frequency of E^n and lE^n (overlap check), or null
};

template <typename R> __device__ __forceinline__ R dsn_div(R num, float dl);
template <> __device__ __forceinline__ float dsn_div<float>(float num, float dl) { return cpml_div(num, dl); }
template <> __device__ __forceinline__ double dsn_div<double>(double num, float dl) { return num / (double)dl; }

template <typename R>
__device__ __forceinline__ R dsn_psi(R* psi, float b, float c, R diff, float dl, long long q) {
    const R nw = b * psi[q] + dsn_div<R>(c * diff, dl);
    psi[q] = nw;
    return nw;
}

template <typename R>
__device__ __forceinline__ bool dsn_edge(const DsnDev<R>& D, int c, int px, int py, int pz, long long* q) {
    const int x = px - D.eo[c][0], y = py - D.eo[c][1], z = pz - D.eo[c][2];
    if (x < 0 || y < 0 || z < 0 || x >= D.en[c][0] || y >= D.en[c][1] || z >= D.en[c][2]) return false;
    *q = D.eoff[c] + ((long long)z * D.en[c][1] + y) * D.en[c][0] + x;
    return true;
}

// design edge q -> component and storage position
template <typename R>
__device__ __forceinline__ int dsn_edge_pos(const DsnDev<R>& D, long long q, int* px, int* py, int* pz) {
    const int c = q >= D.eoff[2] ? 2 : q >= D.eoff[1] ? 1 : 0;
    const long long r = q - D.eoff[c];
    *px = D.eo[c][0] + (int)(r % D.en[c][0]);
    *py = D.eo[c][1] + (int)((r / D.en[c][0]) % D.en[c][1]);
    *pz = D.eo[c][2] + (int)(r / ((long long)D.en[c][0] * D.en[c][1]));
    return c;
}

// Ga/Gb of E edge c: the design box's own values, else the solver's
// (index-1 vacuum default, uniform table, 4-cell average; ref :2516-2527,
// :2832-2853)
template <typename R>
__device__ inline void dsn_coef(const AemParams& P, const DsnDev<R>& D, int c, int px, int py, int pz, R& ga, R& gb) {
    long long q;
    if (dsn_edge(D, c, px, py, pz, &q)) {
        ga = D.ga[q];
        gb = D.gb[q];
        return;
    }
    int i0 = 0, i1 = 0, i2 = 0, i3 = 0;
    if (!(px == 0 || py == 0 || pz == 0)) {
        const uint8_t* C = P.cell;
        i0 = C[lin(P, px, py, pz)];
        if (c == 0) { i1 = C[lin(P, px, py - 1, pz)]; i2 = C[lin(P, px, py, pz - 1)]; i3 = C[lin(P, px, py - 1, pz - 1)]; }
        else if (c == 1) { i1 = C[lin(P, px - 1, py, pz)]; i2 = C[lin(P, px, py, pz - 1)]; i3 = C[lin(P, px - 1, py, pz - 1)]; }
        else { i1 = C[lin(P, px - 1, py, pz)]; i2 = C[lin(P, px, py - 1, pz)]; i3 = C[lin(P, px - 1, py - 1, pz)]; }
    }
    if (i0 == i1 && i0 == i2 && i0 == i3) {
        ga = (R)P.ucoef[i0].ga[c];
        gb = (R)P.ucoef[i0].gb[c];
        return;
    }
    const AemMaterial *m0 = P.mat + i0, *m1 = P.mat + i1, *m2 = P.mat + i2, *m3 = P.mat + i3;
    const float e = (m0->eps[c] + m1->eps[c] + m2->eps[c] + m3->eps[c]) / 4.0f;
    const float s = (m0->sig[c] + m1->sig[c] + m2->sig[c] + m3->sig[c]) / 4.0f;
    ga = (R)d_ga(s, e, P.dt);
    gb = (R)d_gb(s, e, P.dt);
}

template <typename R> __device__ inline void ga_gb(R s, R e, float dt, R& ga, R& gb);
template <> __device__ inline void ga_gb<float>(float s, float e, float dt, float& ga, float& gb) {
    ga = d_ga(s, e, dt);
    gb = d_gb(s, e, dt);
}
template <> __device__ inline void ga_gb<double>(double s, double e, float dt, double& ga, double& gb) {
    const double ep0 = (double)8.85418782E-12f, t = (double)dt;
    ga = (1.0 - s * t / (2.0 * ep0 * e)) / (1.0 + s * t / (2.0 * ep0 * e));
    gb = (t / (ep0 * e)) / (1.0 + s * t / (2.0 * ep0 * e));
}

// the four cells of edge (c, px, py, pz) in the reference's averaging order
__device__ __forceinline__ void edge_cells(int c, int px, int py, int pz, int cx[4], int cy[4], int cz[4]) {
    for (int t = 0; t < 4; t++) { cx[t] = px; cy[t] = py; cz[t] = pz; }
    if (c == 0) { cy[1] -= 1; cz[2] -= 1; cy[3] -= 1; cz[3] -= 1; }
    else if (c == 1) { cx[1] -= 1; cz[2] -= 1; cx[3] -= 1; cz[3] -= 1; }
    else { cx[1] -= 1; cy[2] -= 1; cx[3] -= 1; cy[3] -= 1; }
}

// eps_r and sigma of cell (px, py, pz) for component c
template <typename R>
__device__ __forceinline__ void cell_val(const AemParams& P, const DsnDev<R>& D, int c, int px, int py, int pz, R& e, R& s) {
    const int x = px - D.lo[0], y = py - D.lo[1], z = pz - D.lo[2];
    const AemMaterial& m = P.mat[P.cell[lin(P, px, py, pz)]];
    if (x >= 0 && y >= 0 && z >= 0 && x < D.n[0] && y < D.n[1] && z < D.n[2]) {
        const long long q = ((long long)z * D.n[1] + y) * D.n[0] + x;
        e = D.eps[q];
        s = D.sig ? D.sig[q] : (R)m.sig[c];
    } else {
        e = (R)m.eps[c];
        s = (R)m.sig[c];
    }
}

// Ga/Gb of every design-box edge from the 4-cell averages (ref :2516-2527)
template <typename R>
__global__ void k_dsn_coef(const __grid_constant__ AemParams P, const __grid_constant__ DsnDev<R> D) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < D.nedge; q += (long long)gridDim.x * blockDim.x) {
        int px, py, pz;
        const int c = dsn_edge_pos(D, q, &px, &py, &pz);
        int cx[4], cy[4], cz[4];
        edge_cells(c, px, py, pz, cx, cy, cz);
        R e[4], s[4];
        for (int t = 0; t < 4; t++) cell_val(P, D, c, cx[t], cy[t], cz[t], e[t], s[t]);
        const R ea = (e[0] + e[1] + e[2] + e[3]) / (R)4, sa = (s[0] + s[1] + s[2] + s[3]) / (R)4;
        R ga, gb;
        ga_gb<R>(sa, ea, P.dt, ga, gb);
        D.ga[q] = ga;
        D.gb[q] = gb;
    }
}

// ---------------------------------------------------------------------------
// forward

template <typename R>
__device__ __forceinline__ R ldg(const R* p) { return __ldg(p); }
__device__ __forceinline__ int ldg_id(const uint8_t* p) { return (int)__ldg(p); }

using DsnTabs = CoefTabs;
__device__ inline void load_tabs(const AemParams& P, DsnTabs& T) { load_coef_tabs(P, T); }

// Ga/Gb of E component c from its four cell ids (ref order), as edge_coef
template <typename R>
__device__ __forceinline__ void coef1(const AemParams& P, const DsnTabs& T, int c, int i0, int i1, int i2, int i3, R& ga, R& gb) {
    if (i0 == i1 && i0 == i2 && i0 == i3) {
        ga = (R)T.ga[i0][c];
        gb = (R)T.gb[i0][c];
        return;
    }
    const float e = (T.eps[i0][c] + T.eps[i1][c] + T.eps[i2][c] + T.eps[i3][c]) / 4.0f;
    const float s = (T.sig[i0][c] + T.sig[i1][c] + T.sig[i2][c] + T.sig[i3][c]) / 4.0f;
    ga = (R)d_ga(s, e, P.dt);
    gb = (R)d_gb(s, e, P.dt);
}

// Ga/Gb of the three E components at one position from the ids of the
// cells (px,py), (px-1,py), (px,py-1), (px-1,py-1) in this plane (a) and the
// plane below (b); unaveraged edges (index 1 on an axis) take vacuum.  The
// design box's own values override (the caller).
template <typename R>
__device__ __forceinline__ void coef3(const AemParams& P, const DsnTabs& T, bool unavg, const int a[4], const int b[4], R ga[3], R gb[3]) {
    const int z = unavg ? 0 : a[0];
    if (unavg || (a[0] == a[1] && a[0] == a[2] && a[0] == a[3] && a[0] == b[0] && a[0] == b[1] && a[0] == b[2] && a[0] == b[3])) {
        for (int c = 0; c < 3; c++) {
            ga[c] = (R)T.ga[z][c];
            gb[c] = (R)T.gb[z][c];
        }
        return;
    }
    coef1(P, T, 0, a[0], a[2], b[0], b[2], ga[0], gb[0]);
    coef1(P, T, 1, a[0], a[1], b[0], b[1], ga[1], gb[1]);
    coef1(P, T, 2, a[0], a[1], a[2], a[3], ga[2], gb[2]);
}

// Each thread marches one (x, y) column through DZCH planes; the values of
// the plane below (E for H, H and cell ids for E) are carried in registers.
// Read-only data goes through the non-coherent path so the loads of the
// next plane can issue ahead of this plane's stores.
template <typename R>
__global__ void __launch_bounds__(256, 4) k_dsn_h(const __grid_constant__ AemParams P, const __grid_constant__ DsnDev<R> D) {
    const int px = blockIdx.x * 32 + threadIdx.x, py = blockIdx.y * 8 + threadIdx.y;
    __shared__ DsnTabs T;
    load_tabs(P, T);
    if (px > P.SX - 2 || py > P.SY - 2) return;
    const R *Ex = D.E[0], *Ey = D.E[1], *Ez = D.E[2];
    R *Hx = D.H[0], *Hy = D.H[1], *Hz = D.H[2];
    const int i = px + 1, j = py + 1;
    const float DB = P.DB, dhx = P.den_h[0][i - 1], dhy = P.den_h[1][j - 1];
    const int qx_lo = (i <= P.npml[0][0] - 1) ? i : 0, qx_hi = (i >= P.X + 1 - P.npml[0][1]) ? P.X - i : 0;
    const int qy_lo = (j <= P.npml[1][0] - 1) ? j : 0, qy_hi = (j >= P.Y + 1 - P.npml[1][1]) ? P.Y - j : 0;
    const bool colpml = qx_lo || qx_hi || qy_lo || qy_hi;
    const long long PX = P.PX, PL = P.plane;
    const int pz0 = blockIdx.z * DZCH, pz_end = min(P.SZ - 2, pz0 + DZCH - 1);
    long long c = lin(P, px, py, pz0);
    R ex = ldg(Ex + c), ey = ldg(Ey + c);
    // the loads of a plane: issued one plane ahead of its arithmetic, so two
    // planes of requests are in flight per thread
    struct Plane {
        R ez, ex_jp, ex_kp, ey_ip, ey_kp, ez_ip, ez_jp, hx, hy, hz;
    };
    auto load = [&](long long cc) {
        Plane p;
        p.ez = ldg(Ez + cc);
        p.ex_jp = ldg(Ex + cc + PX); p.ex_kp = ldg(Ex + cc + PL); p.ey_ip = ldg(Ey + cc + 1); p.ey_kp = ldg(Ey + cc + PL);
        p.ez_ip = ldg(Ez + cc + 1); p.ez_jp = ldg(Ez + cc + PX);
        p.hx = ldg(Hx + cc); p.hy = ldg(Hy + cc); p.hz = ldg(Hz + cc);
        return p;
    };
    Plane cur = load(c);
    for (int pz = pz0; pz <= pz_end; pz++, c += PL) {
        Plane nxt = cur;
        if (pz < pz_end) nxt = load(c + PL);
        const int k = pz + 1;
        const float dhz = P.den_h[2][k - 1];
        const R ez = cur.ez, ex_jp = cur.ex_jp, ex_kp = cur.ex_kp, ey_ip = cur.ey_ip, ey_kp = cur.ey_kp;
        const R ez_ip = cur.ez_ip, ez_jp = cur.ez_jp;
        R hxv = cur.hx, hyv = cur.hy, hzv = cur.hz;
        hxv = hxv + DB * ((ez - ez_jp) * dhy + (ey_kp - ey) * dhz);
        hyv = hyv + DB * ((ez_ip - ez) * dhx + (ex - ex_kp) * dhz);
        hzv = hzv + DB * ((ey - ey_ip) * dhx + (ex_jp - ex) * dhy);
        const int qz_lo = (k <= P.npml[2][0] - 1) ? k : 0, qz_hi = (k >= P.Z + 1 - P.npml[2][1]) ? P.Z - k : 0;
        if (colpml || qz_lo || qz_hi) {
            if (qy_lo) hxv = hxv + DB * dsn_psi<R>(D.ph[0][1][0], T.bh[1][0][qy_lo - 1], T.ch[1][0][qy_lo - 1], ez - ez_jp, P.del[1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]));
            if (qy_hi) hxv = hxv + DB * dsn_psi<R>(D.ph[0][1][1], T.bh[1][1][qy_hi - 1], T.ch[1][1][qy_hi - 1], ez - ez_jp, P.del[1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]));
            if (qz_lo) hxv = hxv + DB * dsn_psi<R>(D.ph[0][2][0], T.bh[2][0][qz_lo - 1], T.ch[2][0][qz_lo - 1], ey_kp - ey, P.del[2], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]));
            if (qz_hi) hxv = hxv + DB * dsn_psi<R>(D.ph[0][2][1], T.bh[2][1][qz_hi - 1], T.ch[2][1][qz_hi - 1], ey_kp - ey, P.del[2], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]));
            if (qx_lo) hyv = hyv + DB * dsn_psi<R>(D.ph[1][0][0], T.bh[0][0][qx_lo - 1], T.ch[0][0][qx_lo - 1], ez_ip - ez, P.del[0], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]));
            if (qx_hi) hyv = hyv + DB * dsn_psi<R>(D.ph[1][0][1], T.bh[0][1][qx_hi - 1], T.ch[0][1][qx_hi - 1], ez_ip - ez, P.del[0], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]));
            if (qz_lo) hyv = hyv + DB * dsn_psi<R>(D.ph[1][2][0], T.bh[2][0][qz_lo - 1], T.ch[2][0][qz_lo - 1], ex - ex_kp, P.del[2], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]));
            if (qz_hi) hyv = hyv + DB * dsn_psi<R>(D.ph[1][2][1], T.bh[2][1][qz_hi - 1], T.ch[2][1][qz_hi - 1], ex - ex_kp, P.del[2], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]));
            if (qx_lo) hzv = hzv + DB * dsn_psi<R>(D.ph[2][0][0], T.bh[0][0][qx_lo - 1], T.ch[0][0][qx_lo - 1], ey - ey_ip, P.del[0], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]));
            if (qx_hi) hzv = hzv + DB * dsn_psi<R>(D.ph[2][0][1], T.bh[0][1][qx_hi - 1], T.ch[0][1][qx_hi - 1], ey - ey_ip, P.del[0], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]));
            if (qy_lo) hzv = hzv + DB * dsn_psi<R>(D.ph[2][1][0], T.bh[1][0][qy_lo - 1], T.ch[1][0][qy_lo - 1], ex_jp - ex, P.del[1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]));
            if (qy_hi) hzv = hzv + DB * dsn_psi<R>(D.ph[2][1][1], T.bh[1][1][qy_hi - 1], T.ch[1][1][qy_hi - 1], ex_jp - ex, P.del[1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]));
        }
        Hx[c] = hxv;
        Hy[c] = hyv;
        Hz[c] = hzv;
        ex = ex_kp;
        ey = ey_kp;
        cur = nxt;
    }
}

// E update of one component: bulk, then the CPML psi terms of its two
// difference axes (ax1 with d1, ax2 with d2), as k_update_e
template <typename R>
__device__ __forceinline__ R dsn_e1(const AemParams& P, const DsnTabs& T, const DsnDev<R>& D, int comp, R eold, R d1, R d2, float den1,
                                    float den2, R ga, R gb, bool pml, int q1l, int q1h, int q2l, int q2h, int px, int py,
                                    int pz) {
    const R curl = d1 * den1 + d2 * den2;
    R e = ga * eold + gb * curl;
    if (pml) {
        const int ax1 = comp == 0 ? 1 : 0, ax2 = comp == 2 ? 1 : 2;
        if (q1l) e = e + gb * dsn_psi<R>(D.pe[comp][ax1][0], T.be[ax1][0][q1l - 1], T.ce[ax1][0][q1l - 1], d1, P.del[ax1], psi_idx(P, ax1, q1l, px, py, pz, P.npml[ax1][0]));
        if (q1h) e = e + gb * dsn_psi<R>(D.pe[comp][ax1][1], T.be[ax1][1][q1h - 1], T.ce[ax1][1][q1h - 1], d1, P.del[ax1], psi_idx(P, ax1, q1h, px, py, pz, P.npml[ax1][1]));
        if (q2l) e = e + gb * dsn_psi<R>(D.pe[comp][ax2][0], T.be[ax2][0][q2l - 1], T.ce[ax2][0][q2l - 1], d2, P.del[ax2], psi_idx(P, ax2, q2l, px, py, pz, P.npml[ax2][0]));
        if (q2h) e = e + gb * dsn_psi<R>(D.pe[comp][ax2][1], T.be[ax2][1][q2h - 1], T.ce[ax2][1][q2h - 1], d2, P.del[ax2], psi_idx(P, ax2, q2h, px, py, pz, P.npml[ax2][1]));
    }
    return e;
}

template <typename R>
__global__ void __launch_bounds__(256, 4) k_dsn_e(const __grid_constant__ AemParams P, const __grid_constant__ DsnDev<R> D, int slot) {
    const int px = blockIdx.x * 32 + threadIdx.x, py = blockIdx.y * 8 + threadIdx.y;
    __shared__ DsnTabs T;
    load_tabs(P, T);
    if (px > P.SX - 2 || py > P.SY - 2) return;
    const R *Hx = D.H[0], *Hy = D.H[1], *Hz = D.H[2];
    R *Ex = D.E[0], *Ey = D.E[1], *Ez = D.E[2];
    const int i = px + 1, j = py + 1;
    const float dex = P.den_e[0][i - 1], dey = P.den_e[1][j - 1];
    const int qxl = (i >= 2 && i <= P.npml[0][0]) ? i : 0, qxh = (i >= P.X + 1 - P.npml[0][1] && i <= P.X - 1) ? P.X + 1 - i : 0;
    const int qyl = (j >= 2 && j <= P.npml[1][0]) ? j : 0, qyh = (j >= P.Y + 1 - P.npml[1][1] && j <= P.Y - 1) ? P.Y + 1 - j : 0;
    const bool colpml = qxl || qxh || qyl || qyh;
    const bool xok = px >= 1, yok = py >= 1, unavg_col = px == 0 || py == 0;
    const bool coldsn = px >= D.lo[0] && px <= D.lo[0] + D.n[0] && py >= D.lo[1] && py <= D.lo[1] + D.n[1];
    const uint8_t* C = P.cell;
    const long long PX = P.PX, PL = P.plane;
    const int pz0 = blockIdx.z * DZCH, pz_end = min(P.SZ - 2, pz0 + DZCH - 1);
    long long c = lin(P, px, py, pz0);
    int b[4] = {0, 0, 0, 0};
    R hx_m = 0, hy_m = 0;  // Hx, Hy of the plane below
    if (pz0 > 0) {
        const long long cm = c - PL;
        if (!unavg_col) { b[0] = ldg_id(C + cm); b[1] = ldg_id(C + cm - 1); b[2] = ldg_id(C + cm - PX); b[3] = ldg_id(C + cm - 1 - PX); }
        hx_m = ldg(Hx + cm);
        hy_m = ldg(Hy + cm);
    }
    for (int pz = pz0; pz <= pz_end; pz++, c += PL) {
        const int k = pz + 1;
        int a[4] = {0, 0, 0, 0};
        if (!unavg_col) { a[0] = ldg_id(C + c); a[1] = ldg_id(C + c - 1); a[2] = ldg_id(C + c - PX); a[3] = ldg_id(C + c - 1 - PX); }
        const float dez = P.den_e[2][k - 1];
        const int qzl = (k >= 2 && k <= P.npml[2][0]) ? k : 0, qzh = (k >= P.Z + 1 - P.npml[2][1] && k <= P.Z - 1) ? P.Z + 1 - k : 0;
        const bool pml = colpml || qzl || qzh;
        const R hx = ldg(Hx + c), hy = ldg(Hy + c), hz = ldg(Hz + c);
        // the rest of the plane's loads, issued before any update so that a
        // thread waits on one round of memory latency
        const R ex_o = ldg(Ex + c), ey_o = ldg(Ey + c), ez_o = ldg(Ez + c);
        const R hz_jm = yok ? ldg(Hz + c - PX) : R(0), hx_jm = yok ? ldg(Hx + c - PX) : R(0);
        const R hz_im = xok ? ldg(Hz + c - 1) : R(0), hy_im = xok ? ldg(Hy + c - 1) : R(0);
        R ga[3], gb[3];
        coef3(P, T, unavg_col || pz == 0, a, b, ga, gb);
        const bool dsn = coldsn && pz >= D.lo[2] && pz <= D.lo[2] + D.n[2];
        long long q[3] = {-1, -1, -1};
        if (dsn)
            for (int cc = 0; cc < 3; cc++)
                if (dsn_edge(D, cc, px, py, pz, &q[cc])) { ga[cc] = D.ga[q[cc]]; gb[cc] = D.gb[q[cc]]; }
                else q[cc] = -1;
        if (yok && pz >= 1) {
            const R e = dsn_e1(P, T, D, 0, ex_o, hz - hz_jm, hy_m - hy, dey, dez, ga[0], gb[0], pml, qyl, qyh, qzl, qzh, px, py, pz);
            Ex[c] = e;
            if (slot >= 0 && q[0] >= 0) D.rec[slot * D.nedge + q[0]] = e;
        }
        if (xok && pz >= 1) {
            const R e = dsn_e1(P, T, D, 1, ey_o, hz_im - hz, hx - hx_m, dex, dez, ga[1], gb[1], pml, qxl, qxh, qzl, qzh, px, py, pz);
            Ey[c] = e;
            if (slot >= 0 && q[1] >= 0) D.rec[slot * D.nedge + q[1]] = e;
        }
        if (xok && yok) {
            const R e = dsn_e1(P, T, D, 2, ez_o, hy - hy_im, hx_jm - hx, dex, dey, ga[2], gb[2], pml, qxl, qxh, qyl, qyh, px, py, pz);
            Ez[c] = e;
            if (slot >= 0 && q[2] >= 0) D.rec[slot * D.nedge + q[2]] = e;
        }
        hx_m = hx;
        hy_m = hy;
        for (int t = 0; t < 4; t++) b[t] = a[t];
    }
}

// lumped ports on the H half-step (basic ports; loop current, line
// currents, current source), as k_ports_h
template <typename R>
__global__ void k_dsn_ports_h(const __grid_constant__ AemParams P, const __grid_constant__ PortSet S,
                              const __grid_constant__ DsnDev<R> D, int counter) {
    const int tid = threadIdx.x;
    auto H = [&](int comp, int a, int b, int c) { return D.H[comp][lin(P, a - 1, b - 1, c - 1)]; };
    if (tid == 0) {
        for (int n = 0; n < S.n; n++) {
            const PortDev& p = S.p[n];
            R cur = 0;
            const int p1 = p.loc[0], p2 = p.loc[1], p3 = p.loc[2];
            const int d1 = p.size[0] + p1 - 1, d2 = p.size[1] + p2 - 1, d3 = p.size[2] + p3 - 1;
            if (p.dir == 0) {
                for (int a = p1; a <= d1; a++) {
                    for (int b = p2; b <= d2; b++) cur = cur + p.dl[1] * (H(1, a, b, p3 - 1) - H(1, a, b, d3));
                    for (int c = p3; c <= d3; c++) cur = cur + p.dl[2] * (H(2, a, p2, c) - H(2, a, d2 - 1, c));
                }
                cur = cur * (p.sizef[1] * p.sizef[2]) / p.sizef[0];
            } else if (p.dir == 1) {
                for (int b = p2; b <= d2; b++) {
                    for (int a = p1; a <= d1; a++) cur = cur + p.dl[0] * (H(0, a, b, p3) - H(0, a, b, d3 - 1));
                    for (int c = p3; c <= d3; c++) cur = cur + p.dl[2] * (H(2, p1 - 1, b, c) - H(2, d1, b, c));
                }
                cur = cur * (p.sizef[0] * p.sizef[2]) / p.sizef[1];
            } else {
                for (int c = p3; c <= d3; c++) {
                    for (int a = p1; a <= d1; a++) cur = cur + p.dl[0] * (H(0, a, p2 - 1, c) - H(0, a, d2, c));
                    for (int b = p2; b <= d2; b++) cur = cur + p.dl[1] * (H(1, p1, b, c) - H(1, d1 - 1, b, c));
                }
                cur = cur * (p.sizef[0] * p.sizef[1]) / p.sizef[2];
            }
            D.I[n][0] = cur;
        }
    }
    __syncthreads();
    for (int n = 0; n < S.n; n++) {
        const PortDev& p = S.p[n];
        R *I = D.I[n], *V = D.V[n];
        for (int j = 2 + tid; j <= S.P - 1; j += blockDim.x) I[j - 1] = I[j - 1] - p.cI * (V[j] - V[j - 1]);
    }
    __syncthreads();
    if (tid == 0)
        for (int n = 0; n < S.n; n++)
            if (S.p[n].excite) D.I[n][1] = D.I[n][1] - S.p[n].cI * reinterpret_cast<const float*>(S.srcI)[counter - 1];
}

// lumped ports on the E half-step (line voltages, voltage source, port E),
// as k_ports_e; then the probe's DFT term
template <typename R>
__global__ void k_dsn_ports_e(const __grid_constant__ AemParams P, const __grid_constant__ PortSet S,
                              const __grid_constant__ DsnDev<R> D, int counter) {
    const int tid = threadIdx.x;
    for (int n = 0; n < S.n; n++) {
        const PortDev& p = S.p[n];
        R *I = D.I[n], *V = D.V[n];
        for (int j = 2 + tid; j <= S.P - 1; j += blockDim.x) V[j - 1] = V[j - 1] - p.cV * (I[j - 1] - I[j - 2]);
    }
    __syncthreads();
    if (tid != 0) return;
    for (int n = 0; n < S.n; n++)
        if (S.p[n].excite) D.V[n][1] = D.V[n][1] + S.p[n].cS * reinterpret_cast<const float*>(S.srcV)[counter - 1];
    for (int n = 0; n < S.n; n++) {
        const PortDev& p = S.p[n];
        const R e = 1.0f * D.V[n][1] / (p.sizef[p.dir] * p.dl[p.dir]);
        for (int a = p.loc[0]; a <= p.loc[0] + p.size[0] - 1; a++)
            for (int b = p.loc[1]; b <= p.loc[1] + p.size[1] - 1; b++)
                for (int c = p.loc[2]; c <= p.loc[2] + p.size[2] - 1; c++) D.E[p.dir][lin(P, a - 1, b - 1, c - 1)] = e;
    }
    if (D.acc_dft) {
        double s, co;
        sincospi(D.fdt2 * (double)counter, &s, &co);
        const double v = (double)D.E[D.pc][D.pidx];
        D.dft[0] += v * co;
        D.dft[1] -= v * s;
    }
}

// design-box E into record slot `slot` (the state a segment starts from)
template <typename R>
__global__ void k_dsn_record(const __grid_constant__ AemParams P, const __grid_constant__ DsnDev<R> D, int slot) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < D.nedge; q += (long long)gridDim.x * blockDim.x) {
        int px, py, pz;
        const int c = dsn_edge_pos(D, q, &px, &py, &pz);
        D.rec[slot * D.nedge + q] = D.E[c][lin(P, px, py, pz)];
    }
}

// ---------------------------------------------------------------------------
// adjoint

// gradient sums of forward step n: lE^n at the design edges (the adjoint of
// E^n = Ga E^{n-1} + Gb curl^n) times dE^n/dGa = E^{n-1} and
// Gb dE^n/dGb = E^n - Ga E^{n-1}
// With the overlap check on, also the DFTs at the probe frequency of E^n
// (exp(-i w n dt), (pc, ps) = cos, sin of w n dt) and of lE^n (exp(+i w n dt)).
template <typename R>
__global__ void k_adj_grad(const __grid_constant__ AemParams P, const __grid_constant__ DsnDev<R> D, int sn, int sm,
                           double pc, double ps) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < D.nedge; q += (long long)gridDim.x * blockDim.x) {
        int px, py, pz;
        const int c = dsn_edge_pos(D, q, &px, &py, &pz);
        const double lam = (double)D.w[c][lin(P, px, py, pz)] / (double)D.gb[q];
        const double en = (double)D.rec[sn * D.nedge + q], em = (double)D.rec[sm * D.nedge + q];
        D.A[q] += lam * em;
        D.B[q] += lam * (en - (double)D.ga[q] * em);
        if (D.ov) {
            double* o = D.ov + 4 * q;
            o[0] += en * pc;
            o[1] -= en * ps;
            o[2] += lam * pc;
            o[3] += lam * ps;
        }
    }
}

// The gradient sums A, B estimated from the two spectra alone, the
// frequency-domain overlap of adjoint_optimization.py:121-134 restated for
// this engine: for an adjoint field that is a tone at the probe frequency,
// lE^n = Re(a exp(-i w n dt)) with a = 2 L / nwin (L its DFT over the nwin
// steps), so A = sum lE^n E^{n-1} = Re(a z E) and
// B = sum lE^n (E^n - Ga E^{n-1}) = Re(a (1 - Ga z) E), z = exp(-i w dt),
// E the forward field's DFT.  (cw, sw) = cos, sin of w dt.
template <typename R>
__global__ void k_adj_overlap(const __grid_constant__ DsnDev<R> D, double* Ao, double* Bo, double nwin, double cw,
                              double sw) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < D.nedge; q += (long long)gridDim.x * blockDim.x) {
        const double* o = D.ov + 4 * q;
        const double er = o[0], ei = o[1], ar = 2.0 * o[2] / nwin, ai = 2.0 * o[3] / nwin;
        const double ga = (double)D.ga[q];
        // a E
        const double pr = ar * er - ai * ei, pi = ar * ei + ai * er;
        // z = cw - i sw
        Ao[q] = pr * cw + pi * sw;
        Bo[q] = pr - ga * (pr * cw + pi * sw);
    }
}

// probe seed dF/dc^n = 2 Re(conj(D) e^{-i 2 pi f n dt}); port E and the
// line-voltage update transposed
template <typename R>
__global__ void k_adj_ports_e(const __grid_constant__ AemParams P, const __grid_constant__ PortSet S,
                              const __grid_constant__ DsnDev<R> D, int counter) {
    const int tid = threadIdx.x;
    if (tid == 0) {
        double s, co;
        sincospi(D.fdt2 * (double)counter, &s, &co);
        const double g = 2.0 * (D.dft[0] * co - D.dft[1] * s);
        R ga, gb;
        dsn_coef(P, D, D.pc, D.ppx, D.ppy, D.ppz, ga, gb);
        D.w[D.pc][D.pidx] = D.w[D.pc][D.pidx] + gb * (R)g;
        for (int n = 0; n < S.n; n++) {
            const PortDev& p = S.p[n];
            R sum = 0;
            for (int a = p.loc[0]; a <= p.loc[0] + p.size[0] - 1; a++)
                for (int b = p.loc[1]; b <= p.loc[1] + p.size[1] - 1; b++)
                    for (int c = p.loc[2]; c <= p.loc[2] + p.size[2] - 1; c++) {
                        const long long q = lin(P, a - 1, b - 1, c - 1);
                        R pga, pgb;
                        dsn_coef(P, D, p.dir, a - 1, b - 1, c - 1, pga, pgb);
                        sum = sum + D.w[p.dir][q] / pgb;
                        D.w[p.dir][q] = 0;
                    }
            D.lV[n][1] = D.lV[n][1] + sum / (R)(p.sizef[p.dir] * p.dl[p.dir]);
        }
    }
    __syncthreads();
    // V[m] -= cV (I[m] - I[m-1]), m = 1..P-2
    for (int n = 0; n < S.n; n++) {
        const R cV = S.p[n].cV;
        const R *lV = D.lV[n];
        R* lI = D.lI[n];
        for (int q = tid; q <= S.P - 2; q += blockDim.x) {
            R a = 0;
            if (q + 1 <= S.P - 2) a = a + cV * lV[q + 1];
            if (q >= 1) a = a - cV * lV[q];
            lI[q] = lI[q] + a;
        }
    }
}

// line-current update and loop current transposed
template <typename R>
__global__ void k_adj_ports_h(const __grid_constant__ AemParams P, const __grid_constant__ PortSet S,
                              const __grid_constant__ DsnDev<R> D) {
    const int tid = threadIdx.x;
    // I[m] -= cI (V[m+1] - V[m]), m = 1..P-2
    for (int n = 0; n < S.n; n++) {
        const R cI = S.p[n].cI;
        const R* lI = D.lI[n];
        R* lV = D.lV[n];
        for (int q = tid; q <= S.P - 1; q += blockDim.x) {
            R a = 0;
            if (q >= 1 && q <= S.P - 2) a = a + cI * lI[q];
            if (q >= 2) a = a - cI * lI[q - 1];
            lV[q] = lV[q] + a;
        }
    }
    __syncthreads();
    if (tid != 0) return;
    auto add = [&](int comp, int a, int b, int c, R v) {
        const long long q = lin(P, a - 1, b - 1, c - 1);
        D.lH[comp][q] = D.lH[comp][q] + v;
    };
    for (int n = 0; n < S.n; n++) {
        const PortDev& p = S.p[n];
        const int p1 = p.loc[0], p2 = p.loc[1], p3 = p.loc[2];
        const int d1 = p.size[0] + p1 - 1, d2 = p.size[1] + p2 - 1, d3 = p.size[2] + p3 - 1;
        const R g = D.lI[n][0];
        D.lI[n][0] = 0;
        if (p.dir == 0) {
            const R m = g * (R)((p.sizef[1] * p.sizef[2]) / p.sizef[0]);
            for (int a = p1; a <= d1; a++) {
                for (int b = p2; b <= d2; b++) { add(1, a, b, p3 - 1, p.dl[1] * m); add(1, a, b, d3, -(p.dl[1] * m)); }
                for (int c = p3; c <= d3; c++) { add(2, a, p2, c, p.dl[2] * m); add(2, a, d2 - 1, c, -(p.dl[2] * m)); }
            }
        } else if (p.dir == 1) {
            const R m = g * (R)((p.sizef[0] * p.sizef[2]) / p.sizef[1]);
            for (int b = p2; b <= d2; b++) {
                for (int a = p1; a <= d1; a++) { add(0, a, b, p3, p.dl[0] * m); add(0, a, b, d3 - 1, -(p.dl[0] * m)); }
                for (int c = p3; c <= d3; c++) { add(2, p1 - 1, b, c, p.dl[2] * m); add(2, d1, b, c, -(p.dl[2] * m)); }
            }
        } else {
            const R m = g * (R)((p.sizef[0] * p.sizef[1]) / p.sizef[2]);
            for (int c = p3; c <= d3; c++) {
                for (int a = p1; a <= d1; a++) { add(0, a, p2 - 1, c, p.dl[0] * m); add(0, a, d2, c, -(p.dl[0] * m)); }
                for (int b = p2; b <= d2; b++) { add(1, p1, b, c, p.dl[1] * m); add(1, d1 - 1, b, c, -(p.dl[1] * m)); }
            }
        }
    }
}

// CPML part of the adjoint of E edge (comp)'s difference term along axis
// `which` (1: first, 2: second difference axis): (c / dl) times the psi
// adjoint of each E slab the edge lies in along that axis.  Edges the bulk
// loop never updates hold zero adjoints, so no range test is needed.
template <typename R>
__device__ __forceinline__ R pml_d(const AemParams& P, const DsnTabs& T, const DsnDev<R>& D, int comp, int which, int px, int py, int pz) {
    const int ax = which == 1 ? (comp == 0 ? 1 : 0) : (comp == 2 ? 1 : 2);
    const int r = (ax == 0 ? px : ax == 1 ? py : pz) + 1;
    const int N = ax == 0 ? P.X : ax == 1 ? P.Y : P.Z;
    R v = 0;
    const int ql = (r >= 2 && r <= P.npml[ax][0]) ? r : 0, qh = (r >= N + 1 - P.npml[ax][1] && r <= N - 1) ? N + 1 - r : 0;
    if (ql) v = v + dsn_div<R>(T.ce[ax][0][ql - 1] * D.se[comp][ax][0][psi_idx(P, ax, ql, px, py, pz, P.npml[ax][0])], P.del[ax]);
    if (qh) v = v + dsn_div<R>(T.ce[ax][1][qh - 1] * D.se[comp][ax][1][psi_idx(P, ax, qh, px, py, pz, P.npml[ax][1])], P.del[ax]);
    return v;
}

// CPML part of the adjoint of H face (comp)'s difference term along `ax`
template <typename R>
__device__ __forceinline__ R pml_m(const AemParams& P, const DsnTabs& T, const DsnDev<R>& D, int comp, int ax, int px, int py, int pz) {
    const int r = (ax == 0 ? px : ax == 1 ? py : pz) + 1;
    const int N = ax == 0 ? P.X : ax == 1 ? P.Y : P.Z;
    R v = 0;
    const int ql = (r <= P.npml[ax][0] - 1) ? r : 0, qh = (r >= N + 1 - P.npml[ax][1]) ? N - r : 0;
    if (ql) v = v + dsn_div<R>(T.ch[ax][0][ql - 1] * D.sh[comp][ax][0][psi_idx(P, ax, ql, px, py, pz, P.npml[ax][0])], P.del[ax]);
    if (qh) v = v + dsn_div<R>(T.ch[ax][1][qh - 1] * D.sh[comp][ax][1][psi_idx(P, ax, qh, px, py, pz, P.npml[ax][1])], P.del[ax]);
    return v;
}

__device__ __forceinline__ bool e_slab(const AemParams& P, int ax, int r) {
    const int N = ax == 0 ? P.X : ax == 1 ? P.Y : P.Z;
    return (r >= 2 && r <= P.npml[ax][0]) || (r >= N + 1 - P.npml[ax][1] && r <= N - 1);
}
__device__ __forceinline__ bool h_slab(const AemParams& P, int ax, int r) {
    const int N = ax == 0 ? P.X : ax == 1 ? P.Y : P.Z;
    return r >= 1 && ((r <= P.npml[ax][0] - 1) || (r >= N + 1 - P.npml[ax][1] && r <= N - 1));
}

// E half-step transposed, per H face: lH += (E update)^T [w = Gb lE, se];
// then sh = b sh + DB lH on CPML faces.  E update of edge e:
// E_e = Ga E_e + Gb (d1 den1 + d2 den2) (+ Gb psi), so the adjoint of its
// difference d is den w_e (+ c/dl se), scattered to the two faces of d.
template <typename R>
__global__ void __launch_bounds__(256, 4) k_adj_h(const __grid_constant__ AemParams P, const __grid_constant__ DsnDev<R> D) {
    const int px = blockIdx.x * 32 + threadIdx.x, py = blockIdx.y * 8 + threadIdx.y;
    __shared__ DsnTabs T;
    load_tabs(P, T);
    if (px > P.SX - 2 || py > P.SY - 2) return;
    const R *wX = D.w[0], *wY = D.w[1], *wZ = D.w[2];
    R *lHx = D.lH[0], *lHy = D.lH[1], *lHz = D.lH[2];
    const int i = px + 1, j = py + 1;
    const int qx_lo = (i <= P.npml[0][0] - 1) ? i : 0, qx_hi = (i >= P.X + 1 - P.npml[0][1]) ? P.X - i : 0;
    const int qy_lo = (j <= P.npml[1][0] - 1) ? j : 0, qy_hi = (j >= P.Y + 1 - P.npml[1][1]) ? P.Y - j : 0;
    const bool colph = qx_lo || qx_hi || qy_lo || qy_hi;
    // neighbouring E edges in a CPML slab along x / y (this face's edges at
    // px, px+1 and py, py+1)
    const bool pex = e_slab(P, 0, px + 1) || e_slab(P, 0, px + 2), pey = e_slab(P, 1, py + 1) || e_slab(P, 1, py + 2);
    const float dex0 = P.den_e[0][px], dex1 = P.den_e[0][px + 1], dey0 = P.den_e[1][py], dey1 = P.den_e[1][py + 1];
    const float DB = P.DB;
    const long long PX = P.PX, PL = P.plane;
    const int pz0 = blockIdx.z * DZCH, pz_end = min(P.SZ - 2, pz0 + DZCH - 1);
    long long c = lin(P, px, py, pz0);
    R wx0 = ldg(wX + c), wy0 = ldg(wY + c);
    struct Plane {
        R wxk, wyk, wz0, wxj, wyi, wzi, wzj, lx, ly, lz;
    };
    auto load = [&](long long cc) {
        Plane p;
        p.wxk = ldg(wX + cc + PL); p.wyk = ldg(wY + cc + PL); p.wz0 = ldg(wZ + cc);
        p.wxj = ldg(wX + cc + PX); p.wyi = ldg(wY + cc + 1); p.wzi = ldg(wZ + cc + 1); p.wzj = ldg(wZ + cc + PX);
        p.lx = ldg(lHx + cc); p.ly = ldg(lHy + cc); p.lz = ldg(lHz + cc);
        return p;
    };
    Plane cur = load(c);
    for (int pz = pz0; pz <= pz_end; pz++, c += PL) {
        Plane nxt = cur;
        if (pz < pz_end) nxt = load(c + PL);
        const int k = pz + 1;
        const float dez0 = P.den_e[2][pz], dez1 = P.den_e[2][pz + 1];
        const R wxk = cur.wxk, wyk = cur.wyk, wz0 = cur.wz0, wxj = cur.wxj, wyi = cur.wyi, wzi = cur.wzi, wzj = cur.wzj;
        R lx = cur.lx + ((dez0 * wy0 - dez1 * wyk) - (dey0 * wz0 - dey1 * wzj));
        R ly = cur.ly + ((dez1 * wxk - dez0 * wx0) + (dex0 * wz0 - dex1 * wzi));
        R lz = cur.lz + ((dey0 * wx0 - dey1 * wxj) - (dex0 * wy0 - dex1 * wyi));
        if (e_slab(P, 2, pz + 1) || e_slab(P, 2, pz + 2)) {  // z differences: Ey (Hx), Ex (Hy)
            lx = lx + (pml_d(P, T, D, 1, 2, px, py, pz) - pml_d(P, T, D, 1, 2, px, py, pz + 1));
            ly = ly + (pml_d(P, T, D, 0, 2, px, py, pz + 1) - pml_d(P, T, D, 0, 2, px, py, pz));
        }
        if (pey) {  // y differences: Ez (Hx), Ex (Hz)
            lx = lx - (pml_d(P, T, D, 2, 2, px, py, pz) - pml_d(P, T, D, 2, 2, px, py + 1, pz));
            lz = lz + (pml_d(P, T, D, 0, 1, px, py, pz) - pml_d(P, T, D, 0, 1, px, py + 1, pz));
        }
        if (pex) {  // x differences: Ez (Hy), Ey (Hz)
            ly = ly + (pml_d(P, T, D, 2, 1, px, py, pz) - pml_d(P, T, D, 2, 1, px + 1, py, pz));
            lz = lz - (pml_d(P, T, D, 1, 1, px, py, pz) - pml_d(P, T, D, 1, 1, px + 1, py, pz));
        }
        lHx[c] = lx;
        lHy[c] = ly;
        lHz[c] = lz;
        const int qz_lo = (k <= P.npml[2][0] - 1) ? k : 0, qz_hi = (k >= P.Z + 1 - P.npml[2][1]) ? P.Z - k : 0;
        if (colph || qz_lo || qz_hi) {
            auto upd = [&](R* s, float b, long long q, R l) { s[q] = b * s[q] + DB * l; };
            if (qy_lo) upd(D.sh[0][1][0], T.bh[1][0][qy_lo - 1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]), lx);
            if (qy_hi) upd(D.sh[0][1][1], T.bh[1][1][qy_hi - 1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]), lx);
            if (qz_lo) upd(D.sh[0][2][0], T.bh[2][0][qz_lo - 1], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]), lx);
            if (qz_hi) upd(D.sh[0][2][1], T.bh[2][1][qz_hi - 1], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]), lx);
            if (qx_lo) upd(D.sh[1][0][0], T.bh[0][0][qx_lo - 1], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]), ly);
            if (qx_hi) upd(D.sh[1][0][1], T.bh[0][1][qx_hi - 1], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]), ly);
            if (qz_lo) upd(D.sh[1][2][0], T.bh[2][0][qz_lo - 1], psi_idx(P, 2, qz_lo, px, py, pz, P.npml[2][0]), ly);
            if (qz_hi) upd(D.sh[1][2][1], T.bh[2][1][qz_hi - 1], psi_idx(P, 2, qz_hi, px, py, pz, P.npml[2][1]), ly);
            if (qx_lo) upd(D.sh[2][0][0], T.bh[0][0][qx_lo - 1], psi_idx(P, 0, qx_lo, px, py, pz, P.npml[0][0]), lz);
            if (qx_hi) upd(D.sh[2][0][1], T.bh[0][1][qx_hi - 1], psi_idx(P, 0, qx_hi, px, py, pz, P.npml[0][1]), lz);
            if (qy_lo) upd(D.sh[2][1][0], T.bh[1][0][qy_lo - 1], psi_idx(P, 1, qy_lo, px, py, pz, P.npml[1][0]), lz);
            if (qy_hi) upd(D.sh[2][1][1], T.bh[1][1][qy_hi - 1], psi_idx(P, 1, qy_hi, px, py, pz, P.npml[1][1]), lz);
        }
        wx0 = wxk;
        wy0 = wyk;
        cur = nxt;
    }
}

// Adjoint of one E edge through the H half-step.  The adjoint state kept
// per edge is w = Gb lE (Gb > 0 for every material), so lE = Ga lE + g
// becomes w = Ga w + Gb g; then se = b se + w on its CPML slabs
template <typename R>
__device__ __forceinline__ void adj_e1(const AemParams& P, const DsnTabs& T, const DsnDev<R>& D, int comp, long long c, R wold, R g,
                                       R ga, R gb, bool pml, int q1l, int q1h, int q2l, int q2h, int px, int py, int pz) {
    const R wv = ga * wold + gb * g;
    D.w[comp][c] = wv;
    if (pml) {
        const int ax1 = comp == 0 ? 1 : 0, ax2 = comp == 2 ? 1 : 2;
        auto upd = [&](R* s, float b, long long q) { s[q] = b * s[q] + wv; };
        if (q1l) upd(D.se[comp][ax1][0], T.be[ax1][0][q1l - 1], psi_idx(P, ax1, q1l, px, py, pz, P.npml[ax1][0]));
        if (q1h) upd(D.se[comp][ax1][1], T.be[ax1][1][q1h - 1], psi_idx(P, ax1, q1h, px, py, pz, P.npml[ax1][1]));
        if (q2l) upd(D.se[comp][ax2][0], T.be[ax2][0][q2l - 1], psi_idx(P, ax2, q2l, px, py, pz, P.npml[ax2][0]));
        if (q2h) upd(D.se[comp][ax2][1], T.be[ax2][1][q2h - 1], psi_idx(P, ax2, q2h, px, py, pz, P.npml[ax2][1]));
    }
}

// H half-step transposed, per E edge: the H update
// H_f += DB (d1 den1 + d2 den2) (+ DB psi) gives each of the face's two
// differences the adjoint DB den lH_f (+ c/dl sh), gathered here from the
// four faces around the edge
template <typename R>
__global__ void __launch_bounds__(256, 5) k_adj_e(const __grid_constant__ AemParams P, const __grid_constant__ DsnDev<R> D) {
    const int px = blockIdx.x * 32 + threadIdx.x, py = blockIdx.y * 8 + threadIdx.y;
    __shared__ DsnTabs T;
    load_tabs(P, T);
    if (px > P.SX - 2 || py > P.SY - 2) return;
    const R *lHx = D.lH[0], *lHy = D.lH[1], *lHz = D.lH[2];
    const int i = px + 1, j = py + 1;
    const int qxl = (i >= 2 && i <= P.npml[0][0]) ? i : 0, qxh = (i >= P.X + 1 - P.npml[0][1] && i <= P.X - 1) ? P.X + 1 - i : 0;
    const int qyl = (j >= 2 && j <= P.npml[1][0]) ? j : 0, qyh = (j >= P.Y + 1 - P.npml[1][1] && j <= P.Y - 1) ? P.Y + 1 - j : 0;
    const bool colpe = qxl || qxh || qyl || qyh;
    // neighbouring H faces in a CPML slab along x / y (faces at px-1, px and
    // py-1, py)
    const bool phx = h_slab(P, 0, px + 1) || h_slab(P, 0, px), phy = h_slab(P, 1, py + 1) || h_slab(P, 1, py);
    const bool xok = px >= 1, yok = py >= 1, unavg_col = px == 0 || py == 0;
    const bool coldsn = px >= D.lo[0] && px <= D.lo[0] + D.n[0] && py >= D.lo[1] && py <= D.lo[1] + D.n[1];
    const float DB = P.DB;
    const float bx0 = DB * P.den_h[0][px], bxm = xok ? DB * P.den_h[0][px - 1] : 0.0f;
    const float by0 = DB * P.den_h[1][py], bym = yok ? DB * P.den_h[1][py - 1] : 0.0f;
    const uint8_t* C = P.cell;
    const long long PX = P.PX, PL = P.plane;
    const int pz0 = blockIdx.z * DZCH, pz_end = min(P.SZ - 2, pz0 + DZCH - 1);
    long long c = lin(P, px, py, pz0);
    int b[4] = {0, 0, 0, 0};
    R lx_m = 0, ly_m = 0;  // lHx, lHy of the plane below
    if (pz0 > 0) {
        const long long cm = c - PL;
        if (!unavg_col) { b[0] = ldg_id(C + cm); b[1] = ldg_id(C + cm - 1); b[2] = ldg_id(C + cm - PX); b[3] = ldg_id(C + cm - 1 - PX); }
        lx_m = ldg(lHx + cm);
        ly_m = ldg(lHy + cm);
    }
    for (int pz = pz0; pz <= pz_end; pz++, c += PL) {
        const int k = pz + 1;
        int a[4] = {0, 0, 0, 0};
        if (!unavg_col) { a[0] = ldg_id(C + c); a[1] = ldg_id(C + c - 1); a[2] = ldg_id(C + c - PX); a[3] = ldg_id(C + c - 1 - PX); }
        const float bz0 = DB * P.den_h[2][pz], bzm = pz >= 1 ? DB * P.den_h[2][pz - 1] : 0.0f;
        const int qzl = (k >= 2 && k <= P.npml[2][0]) ? k : 0, qzh = (k >= P.Z + 1 - P.npml[2][1] && k <= P.Z - 1) ? P.Z + 1 - k : 0;
        const bool pe = colpe || qzl || qzh;
        const bool phz = h_slab(P, 2, pz + 1) || h_slab(P, 2, pz);
        const R lx = ldg(lHx + c), ly = ldg(lHy + c), lz = ldg(lHz + c);
        // the -x / -y neighbours, issued with the others before any update
        const R lz_jm = yok ? ldg(lHz + c - PX) : R(0), lx_jm = yok ? ldg(lHx + c - PX) : R(0);
        const R lz_im = xok ? ldg(lHz + c - 1) : R(0), ly_im = xok ? ldg(lHy + c - 1) : R(0);
        const R w0 = ldg(D.w[0] + c), w1 = ldg(D.w[1] + c), w2 = ldg(D.w[2] + c);
        R ga[3], gb[3];
        coef3(P, T, unavg_col || pz == 0, a, b, ga, gb);
        if (coldsn && pz >= D.lo[2] && pz <= D.lo[2] + D.n[2])
            for (int cc = 0; cc < 3; cc++) {
                long long q;
                if (dsn_edge(D, cc, px, py, pz, &q)) { ga[cc] = D.ga[q]; gb[cc] = D.gb[q]; }
            }
        if (yok && pz >= 1) {  // Ex: d1 = Hz - Hz[j-1] (y), d2 = Hy[k-1] - Hy (z)
            R g = (bz0 * ly - bzm * ly_m) + (bym * lz_jm - by0 * lz);
            if (phz) g = g + (pml_m(P, T, D, 1, 2, px, py, pz) - pml_m(P, T, D, 1, 2, px, py, pz - 1));
            if (phy) g = g + (pml_m(P, T, D, 2, 1, px, py - 1, pz) - pml_m(P, T, D, 2, 1, px, py, pz));
            adj_e1(P, T, D, 0, c, w0, g, ga[0], gb[0], pe, qyl, qyh, qzl, qzh, px, py, pz);
        }
        if (xok && pz >= 1) {  // Ey: d1 = Hz[i-1] - Hz (x), d2 = Hx - Hx[k-1] (z)
            R g = (bzm * lx_m - bz0 * lx) + (bx0 * lz - bxm * lz_im);
            if (phz) g = g + (pml_m(P, T, D, 0, 2, px, py, pz - 1) - pml_m(P, T, D, 0, 2, px, py, pz));
            if (phx) g = g + (pml_m(P, T, D, 2, 0, px, py, pz) - pml_m(P, T, D, 2, 0, px - 1, py, pz));
            adj_e1(P, T, D, 1, c, w1, g, ga[1], gb[1], pe, qxl, qxh, qzl, qzh, px, py, pz);
        }
        if (xok && yok) {  // Ez: d1 = Hy - Hy[i-1] (x), d2 = Hx[j-1] - Hx (y)
            R g = (by0 * lx - bym * lx_jm) + (bxm * ly_im - bx0 * ly);
            if (phy) g = g + (pml_m(P, T, D, 0, 1, px, py, pz) - pml_m(P, T, D, 0, 1, px, py - 1, pz));
            if (phx) g = g + (pml_m(P, T, D, 1, 0, px - 1, py, pz) - pml_m(P, T, D, 1, 0, px, py, pz));
            adj_e1(P, T, D, 2, c, w2, g, ga[2], gb[2], pe, qxl, qxh, qyl, qyh, px, py, pz);
        }
        lx_m = lx;
        ly_m = ly;
        for (int t = 0; t < 4; t++) b[t] = a[t];
    }
}

// dF/d eps_r and dF/d sigma per design cell: every edge averages its four
// cells, so a cell receives a quarter of each of its 12 edges' derivatives
template <typename R>
__global__ void k_dsn_cellgrad(const __grid_constant__ AemParams P, const __grid_constant__ DsnDev<R> D, float* geps,
                               float* gsig, double scale) {
    const long long ncell = (long long)D.n[0] * D.n[1] * D.n[2];
    const double ep0 = (double)8.85418782E-12f, dt = (double)P.dt;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(q % D.n[0]), y = (int)((q / D.n[0]) % D.n[1]), z = (int)(q / ((long long)D.n[0] * D.n[1]));
        const int px = D.lo[0] + x, py = D.lo[1] + y, pz = D.lo[2] + z;
        double ge = 0.0, gs = 0.0;
        for (int c = 0; c < 3; c++)
            for (int t = 0; t < 4; t++) {
                const int a = t & 1, b = t >> 1;
                const int ex = px + (c == 0 ? 0 : a), ey = py + (c == 0 ? a : c == 1 ? 0 : b), ez = pz + (c == 2 ? 0 : b);
                long long e;
                if (!dsn_edge(D, c, ex, ey, ez, &e)) continue;
                int cx[4], cy[4], cz[4];
                edge_cells(c, ex, ey, ez, cx, cy, cz);
                double ea = 0.0, sa = 0.0;
                for (int u = 0; u < 4; u++) {
                    R ev, sv;
                    cell_val(P, D, c, cx[u], cy[u], cz[u], ev, sv);
                    ea += (double)ev;
                    sa += (double)sv;
                }
                ea /= 4.0;
                sa /= 4.0;
                const double qd = ep0 * ea + sa * dt / 2.0, q2 = qd * qd;
                const double Ae = D.A[e], Be = D.B[e] / (double)D.gb[e];
                ge += (Ae * (ep0 * sa * dt / q2) + Be * (-dt * ep0 / q2)) / 4.0;
                gs += (Ae * (-ep0 * ea * dt / q2) + Be * (-dt * dt / (2.0 * q2))) / 4.0;
            }
        if (geps) geps[q] = (float)(scale * ge);
        if (gsig) gsig[q] = (float)(scale * gs);
    }
}

// ---------------------------------------------------------------------------

template <typename R>
class DsnImpl : public DesignRun {
   public:
    DsnImpl(const std::string& inputs, const std::string& outdir, const int lo[3], const int n[3]);
    ~DsnImpl() override;
    void set_probe(int comp, int i, int j, int k, double freq_hz) override;
    void set_design(const float* eps, const float* sig) override;
    double forward(int checkpoint_every, double dft[2]) override;
    void gradient(float* geps, float* gsig, double scale) override;
    void set_overlap(bool on) override;
    void gradient_overlap(float* geps, float* gsig, double scale) override;
    void timing(double ms[2], long long launches[2]) const override {
        ms[0] = ms_[0]; ms[1] = ms_[1];
        launches[0] = launches_[0]; launches[1] = launches_[1];
    }
    void get_field(int comp, std::vector<double>& out, int dims[3]) override;
    void* stream() const override { return (void*)st_; }
    size_t device_bytes() const override { return bytes_; }

   private:
    template <typename T>
    T* alloc(size_t n) {
        void* p = nullptr;
        DSN_CUDA(cudaMalloc(&p, n * sizeof(T)));
        bufs_.push_back(p);
        bytes_ += n * sizeof(T);
        DSN_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), st_));
        return (T*)p;
    }
    void step(int n, int slot, int acc, const DsnDev<R>& D, cudaStream_t st);
    void adj_step(int n, int s0, const DsnDev<R>& D);
    void recompute(int seg, const DsnDev<R>& D, cudaStream_t st);
    DsnDev<R> with_rec(int seg) const {
        DsnDev<R> d = D_;
        d.rec = rec_[seg & 1];
        return d;
    }
    cudaEvent_t seg_event(size_t q) {
        while (seg_ev_.size() <= q) {
            cudaEvent_t e;
            DSN_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            seg_ev_.push_back(e);
        }
        return seg_ev_[q];
    }
    void zero(const std::vector<std::pair<void*, size_t>>& v) {
        for (auto& a : v) DSN_CUDA(cudaMemsetAsync(a.first, 0, a.second, st_));
    }
    dim3 vgrid() const { return dim3((P_.SX + 31) / 32, (P_.SY + 7) / 8, (P_.SZ + DZCH - 1) / DZCH); }
    unsigned egrid(long long n) const { return (unsigned)std::max(1LL, std::min((n + 255) / 256, 148LL * 16)); }

    // device scratch released at scope exit
    struct Scratch {
        void* p = nullptr;
        explicit Scratch(size_t bytes) { DSN_CUDA(cudaMalloc(&p, bytes)); }
        ~Scratch() { cudaFree(p); }
        Scratch(const Scratch&) = delete;
        Scratch& operator=(const Scratch&) = delete;
    };

    std::unique_ptr<Solver> s_;
    AemParams P_{};
    PortSet S_{};
    DsnDev<R> D_{};
    cudaStream_t st_ = nullptr;
    std::vector<void*> bufs_;
    size_t bytes_ = 0;
    std::vector<std::pair<void*, size_t>> state_, adj_;  // forward state; adjoint state
    size_t state_bytes_ = 0;
    int steps_ = 0;
    double* ov_buf_ = nullptr;  // overlap check: the two spectra per design edge
    double* ov_ab_ = nullptr;   // overlap check: A, B estimated from them
    bool ov_ready_ = false;
    bool probe_set_ = false, design_set_ = false;
    // checkpoints of the last forward()
    int K_ = 0, nseg_ = 0;
    char* ck_ = nullptr;
    size_t ck_cap_ = 0;
    // design-box E records of one segment, two buffers: the adjoint sweep of
    // one segment reads one while the next segment is recomputed into the
    // other on the side stream
    R* rec_[2] = {nullptr, nullptr};
    size_t rec_cap_ = 0;     // slots allocated per buffer
    cudaStream_t sb_ = nullptr;
    std::vector<cudaEvent_t> seg_ev_;
    bool ready_ = false;     // forward() with checkpoints since set_design
    bool last_recorded_ = false;
    double* dft_ = nullptr;
    R* sig_buf_ = nullptr;
    double ms_[2] = {0, 0};
    long long launches_[2] = {0, 0};
    cudaEvent_t ev_[2] = {nullptr, nullptr};
};

template <typename R>
DsnImpl<R>::DsnImpl(const std::string& inputs, const std::string& outdir, const int lo[3], const int n[3]) {
    s_.reset(new Solver(inputs, false, outdir));
    const Solver& s = *s_;
    P_ = s.params();
    S_ = s.ports();
    st_ = s.stream();
    const Deck& d = s.deck();
    steps_ = d.steps;
    if (P_.per[0] || P_.per[1] || P_.per[2]) throw std::invalid_argument("design gradient: periodic axes are not supported");
    if (P_.tfsf_on) throw std::invalid_argument("design gradient: the deck must be driven by a lumped port, not a plane wave");
    if (P_.nsheet || P_.has_drude) throw std::invalid_argument("design gradient: sheets and Drude poles are not supported");
    for (int q = 0; q < S_.n; q++)
        if (S_.p[q].gridded) throw std::invalid_argument("design gradient: gridded ports are not supported");
    if (s.port_in_cpml()) throw std::invalid_argument("design gradient: a port reaches a CPML slab");
    const int N[3] = {P_.X, P_.Y, P_.Z};
    for (int a = 0; a < 3; a++) {
        // design edges along a span reference indices lo..lo+n; keep them out
        // of both CPML slabs (E: 2..npml and N+1-npml..N-1)
        if (n[a] < 1 || lo[a] <= P_.npml[a][0] || lo[a] < 2 || lo[a] + n[a] >= N[a] + 1 - P_.npml[a][1] || lo[a] + n[a] > N[a] - 2)
            throw std::invalid_argument("design gradient: the design box must keep out of the CPML slabs and the outer walls");
        D_.lo[a] = lo[a] - 1;
        D_.n[a] = n[a];
    }
    for (int q = 0; q < S_.n; q++) {
        const PortDev& p = S_.p[q];
        bool touch = true;
        for (int a = 0; a < 3; a++)
            if (p.loc[a] + p.size[a] < lo[a] - 1 || p.loc[a] > lo[a] + n[a] + 1) touch = false;
        if (touch) throw std::invalid_argument("design gradient: a port touches the design box");
    }
    long long off = 0;
    for (int c = 0; c < 3; c++) {
        for (int a = 0; a < 3; a++) {
            D_.eo[c][a] = D_.lo[a];
            D_.en[c][a] = a == c ? n[a] : n[a] + 1;
        }
        D_.eoff[c] = off;
        off += (long long)D_.en[c][0] * D_.en[c][1] * D_.en[c][2];
    }
    D_.nedge = off;
    const long long ncell = (long long)n[0] * n[1] * n[2];
    // forward state
    const size_t cells = (size_t)s.model().cells;
    for (int c = 0; c < 3; c++) {
        D_.E[c] = alloc<R>(cells);
        D_.H[c] = alloc<R>(cells);
        D_.lH[c] = alloc<R>(cells);
        D_.w[c] = alloc<R>(cells);
        state_.push_back({D_.E[c], cells * sizeof(R)});
        state_.push_back({D_.H[c], cells * sizeof(R)});
        adj_.push_back({D_.lH[c], cells * sizeof(R)});
        adj_.push_back({D_.w[c], cells * sizeof(R)});
    }
    for (int c = 0; c < 3; c++)
        for (int a = 0; a < 3; a++)
            for (int sd = 0; sd < 2; sd++) {
                if (!P_.psi_e[c][a][sd]) continue;
                const int m = P_.npml[a][sd];
                const size_t e0 = a == 0 ? m : P_.PX, e1 = a == 1 ? m : P_.SY, e2 = a == 2 ? m : P_.SZ;
                const size_t ne = e0 * e1 * e2;
                D_.pe[c][a][sd] = alloc<R>(ne);
                D_.ph[c][a][sd] = alloc<R>(ne);
                D_.se[c][a][sd] = alloc<R>(ne);
                D_.sh[c][a][sd] = alloc<R>(ne);
                state_.push_back({D_.pe[c][a][sd], ne * sizeof(R)});
                state_.push_back({D_.ph[c][a][sd], ne * sizeof(R)});
                adj_.push_back({D_.se[c][a][sd], ne * sizeof(R)});
                adj_.push_back({D_.sh[c][a][sd], ne * sizeof(R)});
            }
    for (int q = 0; q < S_.n; q++) {
        D_.V[q] = alloc<R>(S_.P);
        D_.I[q] = alloc<R>(S_.P);
        D_.lV[q] = alloc<R>(S_.P);
        D_.lI[q] = alloc<R>(S_.P);
        state_.push_back({D_.V[q], S_.P * sizeof(R)});
        state_.push_back({D_.I[q], S_.P * sizeof(R)});
        adj_.push_back({D_.lV[q], S_.P * sizeof(R)});
        adj_.push_back({D_.lI[q], S_.P * sizeof(R)});
    }
    for (auto& a : state_) state_bytes_ += (a.second + 255) / 256 * 256;
    R* eps = alloc<R>(ncell);
    D_.eps = eps;
    D_.sig = nullptr;
    D_.ga = alloc<R>(D_.nedge);
    D_.gb = alloc<R>(D_.nedge);
    D_.A = alloc<double>(D_.nedge);
    D_.B = alloc<double>(D_.nedge);
    dft_ = alloc<double>(2);
    D_.dft = dft_;
    D_.pc = -1;
    DSN_CUDA(cudaEventCreate(&ev_[0]));
    DSN_CUDA(cudaEventCreate(&ev_[1]));
    DSN_CUDA(cudaStreamCreateWithFlags(&sb_, cudaStreamNonBlocking));
    DSN_CUDA(cudaStreamSynchronize(st_));
}

template <typename R>
DsnImpl<R>::~DsnImpl() {
    if (st_) cudaStreamSynchronize(st_);
    for (void* p : bufs_) cudaFree(p);
    if (ck_) cudaFree(ck_);
    if (sb_) cudaStreamSynchronize(sb_);
    for (R* r : rec_)
        if (r) cudaFree(r);
    for (cudaEvent_t e : ev_)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : seg_ev_) cudaEventDestroy(e);
    if (sb_) cudaStreamDestroy(sb_);
}

template <typename R>
void DsnImpl<R>::set_probe(int comp, int i, int j, int k, double freq_hz) {
    const int p[3] = {i - 1, j - 1, k - 1};
    const int N[3] = {P_.X, P_.Y, P_.Z};
    if (comp < 0 || comp > 2 || !(freq_hz > 0)) throw std::invalid_argument("design gradient: bad probe component or frequency");
    for (int a = 0; a < 3; a++) {
        const int r = p[a] + 1;
        if (r < 2 || r > N[a] - 2 || r <= P_.npml[a][0] || r >= N[a] + 1 - P_.npml[a][1])
            throw std::invalid_argument("design gradient: the probe must be an interior E edge outside the CPML slabs");
    }
    bool in = true;
    for (int a = 0; a < 3; a++)
        if (p[a] < D_.eo[comp][a] || p[a] >= D_.eo[comp][a] + D_.en[comp][a]) in = false;
    if (in) throw std::invalid_argument("design gradient: the probe lies on the design box");
    for (int q = 0; q < S_.n; q++) {
        const PortDev& pt = S_.p[q];
        if (pt.dir != comp) continue;
        bool on = true;
        for (int a = 0; a < 3; a++)
            if (p[a] + 1 < pt.loc[a] || p[a] + 1 > pt.loc[a] + pt.size[a] - 1) on = false;
        if (on) throw std::invalid_argument("design gradient: the probe lies on a port");
    }
    D_.pc = comp;
    D_.ppx = p[0];
    D_.ppy = p[1];
    D_.ppz = p[2];
    D_.pidx = ((long long)p[2] * P_.SY + p[1]) * P_.PX + p[0];
    D_.fdt2 = 2.0 * freq_hz * (double)P_.dt;
    probe_set_ = true;
}

template <typename R>
__global__ void k_to_r(const float* in, R* out, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        out[q] = (R)in[q];
}

template <typename R>
void DsnImpl<R>::set_design(const float* eps, const float* sig) {
    if (!eps) throw std::invalid_argument("design gradient: eps is required");
    const long long ncell = (long long)D_.n[0] * D_.n[1] * D_.n[2];
    if (sig && !D_.sig) sig_buf_ = alloc<R>(ncell);
    Scratch tmp(2 * ncell * sizeof(float));
    float* t = (float*)tmp.p;
    DSN_CUDA(cudaMemcpyAsync(t, eps, ncell * sizeof(float), cudaMemcpyDefault, st_));
    k_to_r<R><<<egrid(ncell), 256, 0, st_>>>(t, (R*)D_.eps, ncell);
    if (sig) {
        DSN_CUDA(cudaMemcpyAsync(t + ncell, sig, ncell * sizeof(float), cudaMemcpyDefault, st_));
        k_to_r<R><<<egrid(ncell), 256, 0, st_>>>(t + ncell, sig_buf_, ncell);
        D_.sig = sig_buf_;
    } else {
        D_.sig = nullptr;
    }
    k_dsn_coef<R><<<egrid(D_.nedge), 256, 0, st_>>>(P_, D_);
    DSN_CUDA(cudaGetLastError());
    DSN_CUDA(cudaStreamSynchronize(st_));
    design_set_ = true;
    ready_ = false;
}

template <typename R>
void DsnImpl<R>::step(int n, int slot, int acc, const DsnDev<R>& Dv, cudaStream_t st) {
    DsnDev<R> D = Dv;
    D.acc_dft = acc;
    const dim3 blk(32, 8);
    k_dsn_h<R><<<vgrid(), blk, 0, st>>>(P_, D);
    k_dsn_ports_h<R><<<1, 256, 0, st>>>(P_, S_, D, n);
    k_dsn_e<R><<<vgrid(), blk, 0, st>>>(P_, D, slot);
    k_dsn_ports_e<R><<<1, 256, 0, st>>>(P_, S_, D, n);
}

template <typename R>
void DsnImpl<R>::adj_step(int n, int s0, const DsnDev<R>& D) {
    const dim3 blk(32, 8);
    if (n < steps_) {
        double pc = 0.0, ps = 0.0;
        if (D.ov) {
            double ph = D_.fdt2 * (double)n;  // phase in half-turns
            ph -= 2.0 * std::floor(0.5 * ph);
            pc = std::cos(M_PI * ph);
            ps = std::sin(M_PI * ph);
        }
        k_adj_grad<R><<<egrid(D.nedge), 256, 0, st_>>>(P_, D, n - s0, n - 1 - s0, pc, ps);
        launches_[1]++;
    }
    k_adj_ports_e<R><<<1, 256, 0, st_>>>(P_, S_, D, n);
    k_adj_h<R><<<vgrid(), blk, 0, st_>>>(P_, D);
    k_adj_ports_h<R><<<1, 256, 0, st_>>>(P_, S_, D);
    k_adj_e<R><<<vgrid(), blk, 0, st_>>>(P_, D);
    launches_[1] += 4;
}

// forward steps of segment `seg` again from its checkpoint, recording the
// design-box E history into D.rec
template <typename R>
void DsnImpl<R>::recompute(int seg, const DsnDev<R>& D, cudaStream_t st) {
    const int s0 = seg * K_, s1 = std::min(s0 + K_, steps_);
    const char* src = ck_ + (size_t)seg * state_bytes_;
    for (auto& a : state_) {
        DSN_CUDA(cudaMemcpyAsync(a.first, src, a.second, cudaMemcpyDeviceToDevice, st));
        src += (a.second + 255) / 256 * 256;
    }
    k_dsn_record<R><<<egrid(D.nedge), 256, 0, st>>>(P_, D, 0);
    launches_[1]++;
    for (int n = s0 + 1; n <= s1; n++) {
        step(n, n - s0, 0, D, st);
        launches_[1] += 4;
    }
}

template <typename R>
double DsnImpl<R>::forward(int K, double dft[2]) {
    if (!probe_set_ || !design_set_) throw std::invalid_argument("design gradient: set the probe and the design first");
    const int N = steps_;
    const bool plain = K < 1;
    if (!plain) {
        K = std::min(K, N);
        const int nseg = (N + K - 1) / K;
        const size_t need_ck = (size_t)nseg * state_bytes_, need_rec = (size_t)(K + 1) * D_.nedge * sizeof(R);
        if (need_ck > ck_cap_) {
            if (ck_) cudaFree(ck_);
            ck_ = nullptr;
            ck_cap_ = 0;
            DSN_CUDA(cudaMalloc(&ck_, need_ck));
            ck_cap_ = need_ck;
        }
        if ((size_t)(K + 1) > rec_cap_) {
            for (R*& r : rec_) {
                if (r) cudaFree(r);
                r = nullptr;
            }
            rec_cap_ = 0;
            DSN_CUDA(cudaMalloc(&rec_[0], need_rec));
            DSN_CUDA(cudaMalloc(&rec_[1], need_rec));
            rec_cap_ = K + 1;
        }
        K_ = K;
        nseg_ = nseg;
    }
    const DsnDev<R> D = plain ? D_ : with_rec(nseg_ - 1);
    zero(state_);
    DSN_CUDA(cudaMemsetAsync(dft_, 0, 2 * sizeof(double), st_));
    DSN_CUDA(cudaEventRecord(ev_[0], st_));
    launches_[0] = 0;
    int slot_base = -1;  // first step of the recorded (last) segment
    for (int n = 1; n <= N; n++) {
        if (!plain && (n - 1) % K == 0) {
            const int s = (n - 1) / K;
            char* dst = ck_ + (size_t)s * state_bytes_;
            for (auto& a : state_) {
                DSN_CUDA(cudaMemcpyAsync(dst, a.first, a.second, cudaMemcpyDeviceToDevice, st_));
                dst += (a.second + 255) / 256 * 256;
            }
            if (s == nseg_ - 1) {
                slot_base = n - 1;
                k_dsn_record<R><<<egrid(D.nedge), 256, 0, st_>>>(P_, D, 0);
                launches_[0]++;
            }
        }
        step(n, slot_base >= 0 ? n - slot_base : -1, 1, D, st_);
        launches_[0] += 4;
    }
    DSN_CUDA(cudaEventRecord(ev_[1], st_));
    DSN_CUDA(cudaGetLastError());
    double h[2];
    DSN_CUDA(cudaMemcpyAsync(h, dft_, sizeof h, cudaMemcpyDeviceToHost, st_));
    DSN_CUDA(cudaStreamSynchronize(st_));
    float t = 0;
    DSN_CUDA(cudaEventElapsedTime(&t, ev_[0], ev_[1]));
    ms_[0] = t;
    if (dft) { dft[0] = h[0]; dft[1] = h[1]; }
    ready_ = !plain;
    last_recorded_ = !plain;
    return h[0] * h[0] + h[1] * h[1];
}

// The adjoint sweeps segments last to first on the run's stream.  Segment
// s-1 is recomputed on the side stream while segment s is swept: the sweep
// reads only its record buffer, the recompute writes the forward state and
// the other buffer.  Events order each recompute after the sweep that last
// read its buffer, and each sweep after its recompute.  The two streams'
// launches are enqueued in alternating chunks, so neither waits behind the
// other's backlog in the launch queue.
template <typename R>
void DsnImpl<R>::gradient(float* geps, float* gsig, double scale) {
    if (!ready_) throw std::invalid_argument("design gradient: run forward() with checkpoints first");
    const int N = steps_, K = K_, S = nseg_;
    constexpr int CHUNK = 16;  // steps per stream per enqueue turn
    zero(adj_);
    DSN_CUDA(cudaMemsetAsync(D_.A, 0, D_.nedge * sizeof(double), st_));
    DSN_CUDA(cudaMemsetAsync(D_.B, 0, D_.nedge * sizeof(double), st_));
    if (D_.ov) DSN_CUDA(cudaMemsetAsync(D_.ov, 0, 4 * D_.nedge * sizeof(double), st_));
    ov_ready_ = false;
    DSN_CUDA(cudaEventRecord(ev_[0], st_));
    DSN_CUDA(cudaStreamWaitEvent(sb_, ev_[0], 0));
    launches_[1] = 0;
    auto ev_sweep = [&](int s) { return seg_event(2 * (size_t)s); };
    auto ev_rec = [&](int s) { return seg_event(2 * (size_t)s + 1); };
    if (!last_recorded_) {
        recompute(S - 1, with_rec(S - 1), st_);  // same stream as its sweep
        DSN_CUDA(cudaEventRecord(ev_rec(S - 1), st_));
        DSN_CUDA(cudaStreamWaitEvent(sb_, ev_rec(S - 1), 0));  // both write the forward state
    }
    for (int s = S - 1; s >= 0; s--) {
        // recompute of segment s-1 on the side stream
        const int r = s - 1;
        const DsnDev<R> Dr = with_rec(r >= 0 ? r : 0);
        int rn = 0, r1 = -1, r0 = 0;
        if (r >= 0) {
            if (s + 1 < S) DSN_CUDA(cudaStreamWaitEvent(sb_, ev_sweep(s + 1), 0));
            r0 = r * K;
            r1 = std::min(r0 + K, N);
            const char* src = ck_ + (size_t)r * state_bytes_;
            for (auto& a : state_) {
                DSN_CUDA(cudaMemcpyAsync(a.first, src, a.second, cudaMemcpyDeviceToDevice, sb_));
                src += (a.second + 255) / 256 * 256;
            }
            k_dsn_record<R><<<egrid(Dr.nedge), 256, 0, sb_>>>(P_, Dr, 0);
            launches_[1]++;
            rn = r0 + 1;
        }
        // sweep of segment s on the run's stream, after its recompute
        if (s < S - 1) DSN_CUDA(cudaStreamWaitEvent(st_, ev_rec(s), 0));
        const DsnDev<R> Da = with_rec(s);
        const int s0 = s * K;
        int an = std::min(s0 + K, N);
        while (rn <= r1 || an > s0) {
            for (int q = 0; q < CHUNK && rn <= r1; q++, rn++) {
                step(rn, rn - r0, 0, Dr, sb_);
                launches_[1] += 4;
            }
            for (int q = 0; q < CHUNK && an > s0; q++, an--) adj_step(an, s0, Da);
        }
        if (r >= 0) DSN_CUDA(cudaEventRecord(ev_rec(r), sb_));
        DSN_CUDA(cudaEventRecord(ev_sweep(s), st_));
    }
    last_recorded_ = false;  // earlier segments' recomputes overwrote the records
    const long long ncell = (long long)D_.n[0] * D_.n[1] * D_.n[2];
    Scratch buf(2 * ncell * sizeof(float));
    float* out = (float*)buf.p;
    k_dsn_cellgrad<R><<<egrid(ncell), 256, 0, st_>>>(P_, D_, out, out + ncell, scale);
    launches_[1]++;
    DSN_CUDA(cudaEventRecord(ev_[1], st_));
    DSN_CUDA(cudaGetLastError());
    if (geps) DSN_CUDA(cudaMemcpyAsync(geps, out, ncell * sizeof(float), cudaMemcpyDefault, st_));
    if (gsig) DSN_CUDA(cudaMemcpyAsync(gsig, out + ncell, ncell * sizeof(float), cudaMemcpyDefault, st_));
    DSN_CUDA(cudaStreamSynchronize(st_));
    DSN_CUDA(cudaStreamSynchronize(sb_));
    float t = 0;
    DSN_CUDA(cudaEventElapsedTime(&t, ev_[0], ev_[1]));
    ms_[1] = t;
    ov_ready_ = D_.ov != nullptr;
}

template <typename R>
void DsnImpl<R>::set_overlap(bool on) {
    if (on && !ov_buf_) {
        ov_buf_ = alloc<double>(4 * (size_t)D_.nedge);
        ov_ab_ = alloc<double>(2 * (size_t)D_.nedge);
    }
    D_.ov = on ? ov_buf_ : nullptr;
    ov_ready_ = false;
}

template <typename R>
void DsnImpl<R>::gradient_overlap(float* geps, float* gsig, double scale) {
    if (!ov_ready_)
        throw std::invalid_argument("design gradient: enable the overlap check, then run forward() and gradient()");
    const double wdt = M_PI * D_.fdt2;  // w dt
    DsnDev<R> Dv = D_;
    Dv.A = ov_ab_;
    Dv.B = ov_ab_ + D_.nedge;
    k_adj_overlap<R><<<egrid(D_.nedge), 256, 0, st_>>>(D_, Dv.A, Dv.B, (double)(steps_ - 1), std::cos(wdt), std::sin(wdt));
    const long long ncell = (long long)D_.n[0] * D_.n[1] * D_.n[2];
    Scratch buf(2 * ncell * sizeof(float));
    float* out = (float*)buf.p;
    k_dsn_cellgrad<R><<<egrid(ncell), 256, 0, st_>>>(P_, Dv, out, out + ncell, scale);
    DSN_CUDA(cudaGetLastError());
    if (geps) DSN_CUDA(cudaMemcpyAsync(geps, out, ncell * sizeof(float), cudaMemcpyDefault, st_));
    if (gsig) DSN_CUDA(cudaMemcpyAsync(gsig, out + ncell, ncell * sizeof(float), cudaMemcpyDefault, st_));
    DSN_CUDA(cudaStreamSynchronize(st_));
}

template <typename R>
void DsnImpl<R>::get_field(int comp, std::vector<double>& out, int dims[3]) {
    if (comp < 0 || comp > 5) throw std::invalid_argument("design gradient: field component must be 0..5");
    static const int ext[6][3] = {{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {0, -1, -1}, {-1, 0, -1}, {-1, -1, 0}};
    const int N[3] = {P_.X, P_.Y, P_.Z};
    for (int a = 0; a < 3; a++) dims[a] = N[a] + ext[comp][a];
    const size_t cells = (size_t)s_->model().cells;
    std::vector<R> all(cells);
    DSN_CUDA(cudaMemcpyAsync(all.data(), comp < 3 ? D_.E[comp] : D_.H[comp - 3], cells * sizeof(R), cudaMemcpyDeviceToHost, st_));
    DSN_CUDA(cudaStreamSynchronize(st_));
    out.assign((size_t)dims[0] * dims[1] * dims[2], 0.0);
    const int S[3] = {P_.SX, P_.SY, P_.SZ};
    for (int k = 1; k <= dims[2] && k <= S[2]; k++)
        for (int j = 1; j <= dims[1] && j <= S[1]; j++)
            for (int i = 1; i <= dims[0] && i <= S[0]; i++)
                out[((size_t)(k - 1) * dims[1] + (j - 1)) * dims[0] + (i - 1)] =
                    (double)all[((size_t)(k - 1) * P_.SY + (j - 1)) * P_.PX + (i - 1)];
}

}  // namespace

DesignRun* DesignRun::create(const std::string& inputs_path, const std::string& outdir, const int lo[3], const int n[3],
                             int precision) {
    if (precision == 4) return new DsnImpl<float>(inputs_path, outdir, lo, n);
    if (precision == 8) return new DsnImpl<double>(inputs_path, outdir, lo, n);
    throw std::invalid_argument("design gradient: precision must be 4 (FP32) or 8 (FP64)");
}

}  // namespace aem
