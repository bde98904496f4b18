// aem_types.h -- host/device data layout of the B200 FDTD solver.
//
// Index conventions.  Every field component keeps the reference's 1-based
// Yee indices (main_fdtd/fdtd_solver.f90:3908-3913): Ex(X-1,Y,Z), Ey(X,Y-1,Z),
// Ez(X,Y,Z-1), Hx(X,Y-1,Z-1), Hy(X-1,Y,Z-1), Hz(X-1,Y-1,Z) with
// X = nx+1+pbc_x (and likewise Y, Z).  On the device all six components share
// one padded storage shape [SZ][SY][PX] (x fastest, rows 128-byte aligned);
// reference index i lives at storage position i-1.
//   - non-periodic axis of size N: positions 0..N-1.  Position N-1 holds the
//     outer PEC wall of tangential E (never written, stays 0).
//   - periodic axis: the reference models one duplicated layer (index N-1 is a
//     copy of index 1, fdtd_solver.f90:1316-1318, :5377-5433, :6672-6806).
//     Here the axis is stored once with n = N-2 positions and neighbour reads
//     wrap; for kmax a wrapped read carries the Bloch phase exp(-+ikL).
// Cell material IDs (uint8, 0 = vacuum) use the same storage positions as
// the fields (cell (i,j,k) at position (i-1,j-1,k-1)).
#pragma once
#include <stdint.h>

#ifndef AEM_MAX_MATERIALS
#define AEM_MAX_MATERIALS 256
#endif
#define AEM_MAX_POLES 6
#define AEM_MAX_PML 64
#define AEM_MAX_SHEET_PLANES 16
#define AEM_MAX_PORTS 16
#define AEM_MAX_FF_ANGLES 4096
#define AEM_MAX_DFT_FREQS 4096
#define AEM_MAX_DFT_SERIES (4 + AEM_MAX_PORTS)
#define AEM_MAX_PROBES 64

// Per-material constants (cell properties), ref materials_properties(:,:,:)
struct AemMaterial {
    float eps[3];
    float sig[3];
    float wp[AEM_MAX_POLES][3];   // plasma frequency per pole and axis
    float gam[AEM_MAX_POLES][3];  // collision frequency per pole and axis
};

// Coefficients of an E edge whose four neighbouring cells hold the same
// material: Ga/Gb per axis and Drude Ja/Jb per pole and axis.  Computed on
// the host with the reference's own 4-term average so the fast path equals
// the general formula bit for bit.
struct AemUniformCoef {
    float ga[3], gb[3];
    float ja[AEM_MAX_POLES][3], jb[AEM_MAX_POLES][3];
};

// One sheet plane: all sheets whose normal is `axis` at reference index
// `pos`.  2-D arrays are over the two in-plane axes (a = first, b = second
// of (y,z) / (x,z) / (x,y)), storage positions, pitch `pa`.
struct AemSheetPlane {
    int axis, pos;       // normal axis 0/1/2, storage position along it
    int pa, na, nb;      // pitch and extents of the 2-D arrays
    // normal component: mask + E_special update coefficients
    const uint8_t* nmask;  // 1 where sheet_sig>0 .or. sheet_ep>1 (ref :4496)
    const float* sa;       // E_special Ga, ref :5723-5726
    const float* sb;       // E_special Gb
    void* es;              // E_special (normal component), in place; complex when kmax
    // tangential components: Ga/Gb overrides (ref :2922-3120)
    const uint8_t* tmask;  // bit0: first tangential overridden, bit1: second
    const float* ga1; const float* gb1;
    const float* ga2; const float* gb2;
};

// All constants one step needs.  Passed to every kernel as a
// __grid_constant__ parameter, so a captured CUDA graph carries it.
struct AemParams {
    // grid
    int X, Y, Z;            // reference sizes (nx+1+pbc)
    int per[3];             // periodic flags
    int SX, SY, SZ;         // storage extents (N, or N-2 when periodic)
    int PX;                 // x pitch (elements)
    long long plane;        // PX*SY
    int kmax;               // complex fields + Bloch phases
    float bloch_re[3], bloch_im[3];  // exp(+i k (N-2) d) per axis (kmax)
    float DB;               // dt/mu0
    float dt, del[3];
    // fields (float*, or interleaved complex when kmax) and cell IDs
    void* E[3];
    void* H[3];
    const uint8_t* cell;
    // CPML thickness in surfaces (reference nxPML_1 ...), [axis][low/high]
    int npml[3][2];
    // den_e*/den_h* by axis; element idx-1 holds den(idx)
    const float* den_e[3];
    const float* den_h[3];
    // CPML b/c, [axis][side][q-1]
    float be[3][2][AEM_MAX_PML], ce[3][2][AEM_MAX_PML];
    float bh[3][2][AEM_MAX_PML], ch[3][2][AEM_MAX_PML];
    // psi arrays [field comp][slab axis][side] (complex when kmax)
    void* psi_h[3][3][2];
    void* psi_e[3][3][2];
    // materials
    int nmat, npoles, has_drude;
    const AemMaterial* mat;
    const AemUniformCoef* ucoef;
    // Drude boxes (reference indices kmin,kmax,jmin,jmax,imin,imax) and the
    // per-component current arrays over the box in storage positions:
    // origin, extents, layout [pole][z][y][x]
    int dbox[3][6];
    int jorg[3][3], jext[3][3];
    void* jsrc[3];
    // sheets
    int nsheet;
    AemSheetPlane sheet[AEM_MAX_SHEET_PLANES];
    float sheet_thick;
    // TF/SF plane wave (standard solver)
    int tfsf_on, mirror_on;
    int tfsf_sep;  // the TF/SF faces stay clear of every CPML slab: corrected by their own kernels
    int lo[3], hi[3];
    float wall_lo[3], wall_hi[3];
    float t_spread, spread, exp_half, inv_c;
    int pulse_type;
    float WE[2][3], WH[2][3];          // [0] incident, [1] mirrored
    float sc[2][3];                    // sin(th)cos(ph), sin(th)sin(ph), cos(th)
    int delay[2][3];
    float coef_h[3], coef_e[3];        // dt/(mu0*d), dt/(ep0*d)
    // kmax plane source
    int kmax_src_axis, kmax_mode_TE, kmax_mode_TM, k_pl_H, k_pl_E;
    float kcnt[3], knum[3], two_pi_f;
    // 0: update kernels apply bulk and CPML together; 1: bulk only; 2: CPML
    // only (a port inside a CPML slab needs the reference's order: bulk,
    // port half-step, CPML pass)
    int cpml_split;
    // fused H+E step (k_yee): the new fields and H-psi go to these buffers
    // (ping-pong with E/H/psi_h above; the host swaps them after each step)
    void* E2[3];
    void* H2[3];
    void* psi_h2[3][3][2];
    // device counter of fused-step CTAs that gave up a bounded wait (0 = ok)
    int* err;
    // launch shape of the two-kernel update (k_update_h / k_update_e): z
    // planes per CTA and rows (y) per CTA of 32 columns; the autotuner picks
    // them per run and per kernel (the fields do not depend on them)
    int zch_h, ty_h, zch_e, ty_e;
    // graph replay: the step number (1-based) lives in device memory and the
    // kernels read it instead of their `counter` argument (null: eager steps)
    const int* dstep;
};
