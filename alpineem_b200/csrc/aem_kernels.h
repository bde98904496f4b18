// aem_kernels.h -- launch interface of the per-step kernels (each launcher
// returns the number of kernels it launched).
#pragma once
#include <cuda_runtime.h>

#include "aem_types.h"

namespace aem {

// one lumped port on the device (ref ports(:,:,:), Voltage/Current lines)
struct PortDev {
    int gridded, dir, side;
    int loc[3], size[3];        // reference indices / cell counts (ports(i,3..4,:))
    float sizef[3];             // ports(i,4,:) as reals
    int n1, n2;                 // gridded feed extent
    const float* feed;          // (4, n1+1, n2+1) F-order; gridded only
    float feed_norm;            // mode normalisation (ref :4948-4954), host computed
    float cI, cV, cS;           // (1/L)(dt/d), (1/C)(dt/d), (1/sqrt(CL))(dt/d)
    float dl[3];                // del_x, del_y, del_z
    void* V;                    // Voltage(1..P), complex when kmax
    void* I;                    // Current(1..P-1)
    void* vout;                 // Voltage_out(1..steps)
    int excite;                 // this port is the excitation port
};

struct PortSet {
    int n, P;                   // number of ports, port_array_size
    PortDev p[AEM_MAX_PORTS];
    const void* srcI;           // E_or_V_1D(amp, n, 0) per step (index n-1)
    const void* srcV;           // E_or_V_1D(amp, n+0.5, 0.5 d) per step
};

// far-field Huygens box
struct FarFieldDev {
    int nang, len;              // angles, bins per series (len_ff + 2)
    int lo[3], hi[3];           // ff_xlow.. (reference indices)
    int has[3];                 // faces present per axis (non-periodic)
    int ic, jc, kc;
    float r_relay, c_dt;        // r_for_time_relay, c*dt
    float fac[3];               // area/(4 pi dt c) per face normal
    float wall_lo[3], wall_hi[3];
    const float* ang;           // per angle: sin(th), cos(th), sin(ph), cos(ph)
    void* cur[3][2];            // per face normal / side: the 4 current components of the last step
    long long face_n[3];        // cells per face of that normal
    void* UW;                   // [6][nang][len] FP64: Wx,Wy,Wz,Ux,Uy,Uz (kmax: a real plane, then an imaginary one)
    int mirror;                 // image-ground-plane pass
    float mir_off[3], use_mir[3], M_mir[3], J_mir[3];
    float kc3[3];               // kmax: k_count for Bloch-phase removal
    // time-batched binning: the differences of tb steps are kept and binned
    // together; constant-k runs bin their real and imaginary parts as two
    // planes of dtile and UW, each as an FP32 run's
    int tb;
    int nvang;                  // virtual angles: nang * (1 + mirror), image pass second
    int tiles_u[3], tiles_v[3]; // 32x32 tiles per face of each normal
    long long tile0[7];         // first tile of face (a, s) at index 2a+s
    int ntiles;                 // tiles over all six faces (tile0[6])
    const float* kf;            // [nvang][3][2][3]: K0, Ku, Kv of the retarded-time offset tf(u, v)
    // deterministic tiled binning (FP32 path, aem_ffbin.cu)
    float* dtile;               // [tile][FF_SLOTS][4][1024] current differences; slot 0: the step before the batch
    int nvc;                    // binned (canonical) virtual angles
    const int* vlist;           // [nvc] their virtual-angle ids
    int hs;                     // bins of one (tile, angle) window (lanes included)
    int group;                  // angles per binning CTA (a multiple of the warps)
    int ngrp;                   // angle groups: ceil(nvc / group)
    const int* kb;              // [tile][nvc] window base: the lowest bin offset any cell of the tile reaches
    float* part;                // [tile][nvc][4][hs] window sums of one batch (U1, U2, W1, W2)
    const int* srt;             // [nvc][6][maxt] tiles of each face sorted by (kb, tile)
    const int* srtkb;           // the same layout: kb of each sorted tile
    int maxt;                   // tiles of the largest face
    int nangc;                  // canonical angles (reduction CTAs)
    const int* clist;           // [nangc][4]: angle, j of pass 0, j of pass 1 (-1: none), unused
    const int* crange;          // [nangc][2]: bin offsets [lo, hi) the angle's windows cover
    int* err;                   // count of contributions that fell outside a window (must stay 0)
};

constexpr int FF_TB = 32;     // steps per far-field batch (one per warp lane)
constexpr int FF_TILE = 32;   // face tile edge of the batched binning
constexpr int FF_SLOTS = 34;  // difference slots per tile: carry, 32 steps, one spare

// per-step output taps
struct TapDev {
    int plane_sum;              // standard unit-cell plane sums
    int axis;                   // normal of the reflection/transmission planes
    float w1, w2;               // projection weights (see plane_sum kernel)
    void* refl;                 // per step
    void* trans;
    void* refl_tm;              // kmax: TM sums (refl/trans above are TE)
    void* trans_tm;
    float knum[3];
    int ff_pc;                  // phase-centre sample
    int ic, jc, kc;
    void* pc[6];                // Ex,Ey,Ez,Hx,Hy,Hz per step (+1)
    // point probes (extension `probe i j k`): the phase-centre sample's
    // cell-centred Ex, Ey, Ez at each probe cell, every step
    int nprobe;
    int prb_idx[AEM_MAX_PROBES][3];
    void* prb;                  // [probe][component][step]
    int video;                  // 2-D slice export
    int slice_dir, slice_loc, v1, v2;
    void* vid[6];               // Ex,Hx,Ey,Hy,Ez,Hz each (v1, v2, steps)
    // on-the-fly spectra: X[s][f] += x_s[m] exp(-i 2 pi f m dt) every step
    // (m = step - 1), FP64 sums with Kahan compensation
    int ndft, nser;             // frequencies, series
    double dft_dt;
    const double* dft_f;        // [ndft] Hz
    double* dft_acc;            // [nser][ndft][re, im]
    double* dft_cmp;            // compensations, same layout
    const void* ser[AEM_MAX_DFT_SERIES];  // per-step samples of each series
};

// the six field arrays (Ex, Ey, Ez, Hx, Hy, Hz) the watchdog scans
struct FieldPtrs {
    const void* p[6];
};
int launch_nonfinite(const FieldPtrs& F, long long n4, int* flag, cudaStream_t s);  // *flag = 1 on a NaN or Inf

int launch_update_h(const AemParams& P, int counter, cudaStream_t s);
int launch_update_e(const AemParams& P, int counter, cudaStream_t s);
int launch_ports_h(const AemParams& P, const PortSet& ps, int counter, cudaStream_t s);
int launch_ports_e(const AemParams& P, const PortSet& ps, int counter, cudaStream_t s);
int launch_ff_currents(const AemParams& P, const FarFieldDev& F, int slot, cudaStream_t s);
// deterministic tiled binning (aem_ffbin.cu): bin `nlanes` steps starting at
// n0 (the differences in slots 1..nlanes, the step before in slot 0), add
// the windows to the FP64 accumulators in a fixed order, then move slot
// `carry` to slot 0 for the next batch (carry < 0: no move).  tail: the
// run's last batch, whose last lane also bins the carried part of the final
// step (the windows need FF_TB + 1 bins beyond the span)
int launch_ff_bin_tiles(const AemParams& P, const FarFieldDev& F, int n0, int nlanes, int carry, cudaStream_t s,
                        bool tail = false);
// window bases kb and the largest window span over all (tile, angle)
int launch_ff_base(const FarFieldDev& F, int* kb, int* span, cudaStream_t s);
size_t ff_tiles_smem(const FarFieldDev& F);  // dynamic shared bytes of one binning CTA
void ff_tiles_prepare();                     // raise the kernel's shared-memory limit (once per device)
// fused H+E step (aem_yee.cu): usable when the deck has none of TF/SF,
// sheets, Drude poles, gridded ports, kmax
bool yee_fused_ok(const AemParams& P, int gridded_ports);
int launch_yee(const AemParams& P, cudaStream_t s);
int launch_yee4(const AemParams& P, cudaStream_t s);  // aem_yee4.cu (no x/y periodicity)
int launch_taps(const AemParams& P, const TapDev& T, const FarFieldDev& F, int counter, int steps, cudaStream_t s);
// full-field export of one step into `out` (6 x n0*n1*n2 values)
int launch_full(const AemParams& P, void* out, const int n[3], cudaStream_t s);
int launch_step_advance(int* d, cudaStream_t s);  // aem_aux.cu: *d += 1 (graph replay)

}  // namespace aem
