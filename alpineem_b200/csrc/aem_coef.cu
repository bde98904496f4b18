// aem_coef.cu -- the run's coefficient tables computed on the GPU in FP64
// (extension `coef_precision 64`).
//
// The reference computes its update coefficients once, in FP32 (Fortran
// default real), except for an FP64 intermediate in the Drude Jb
// (main_fdtd/fdtd_solver.f90:2870-2875):
//   Ga/Gb of every material           :2832-2858   (with Drude :2859-2918)
//   Drude Ja/Jb per pole              :2870-2875
//   CPML b, c and kappa per depth     :3404-3577   (graded sigma, alpha, kappa)
//   den_e / den_h = 1 / (kappa d)     :3584-3666
// With `coef_precision 64` these tables are evaluated on the device in
// FP64 from the same FP32 inputs and rounded to FP32 once at the end, so
// each coefficient is the correctly rounded value of the reference's
// expression instead of the result of a chain of FP32 roundings.  The
// default (reference mode) keeps the host's FP32 evaluation in the
// reference's operation order, which parity with the reference is defined
// on.  Interface edges, whose coefficients the update kernels derive from
// the four neighbouring cells' materials, and sheet overrides are
// unchanged.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "aem_model.h"

namespace aem {

namespace {

struct CoefIn {
    int nmat, npoles, m;
    double dt;
    int npml[3][2];
    int N[3];
    long long den_off[3];  // first den_h value of axis a (den_e follows N[a] + 1 later)
    double dl[3], sig_max[3], alpha_max, kappa_max;
};

constexpr double kEp0d = 8.85418782E-12;

// out layout: per axis a, side s: be[n], ce[n], ke[n+1] (index 1..n), bh, ch,
// kh (index 1..n-1), each AEM_MAX_PML + 1 long
constexpr int CP_STRIDE = AEM_MAX_PML + 1;
__device__ inline float* cp_row(float* out, int a, int s, int which) {
    return out + (((size_t)a * 2 + s) * 6 + which) * CP_STRIDE;
}

__device__ inline double gpow(double g, int m) {
    double p = g;
    for (int q = 1; q < m; q++) p *= g;
    return p;
}

// one thread per (material, axis), per (axis, side, depth) and per
// (axis, grid index) of the den tables
__global__ void k_coef_fp64(const AemMaterial* mats, CoefIn in, AemUniformCoef* uc, float* cpml, float* den) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const double dt = in.dt;
    if (t < in.nmat * 3) {
        const int mi = t / 3, c = t % 3;
        const AemMaterial& am = mats[mi];
        const double e = am.eps[c], s = am.sig[c];
        double tp = 0.0;
        for (int p = 0; p < in.npoles; p++) {
            const double w = am.wp[p][c], g = am.gam[p][c];
            const double ja = (1.0 - g * dt / 2.0) / (1.0 + g * dt / 2.0);
            const double jb = (w * w * kEp0d * dt / 2.0) / (1.0 + g * dt / 2.0);
            uc[mi].ja[p][c] = (float)ja;
            uc[mi].jb[p][c] = (float)jb;
            tp += jb;
        }
        const double st = s + tp;
        uc[mi].ga[c] = (float)((1.0 - st * dt / (2.0 * kEp0d * e)) / (1.0 + st * dt / (2.0 * kEp0d * e)));
        uc[mi].gb[c] = (float)((dt / (kEp0d * e)) / (1.0 + st * dt / (2.0 * kEp0d * e)));
        return;
    }
    int u = t - in.nmat * 3;
    if (u < 3 * 2 * CP_STRIDE) {
        const int a = u / (2 * CP_STRIDE), s = (u / CP_STRIDE) % 2, i = u % CP_STRIDE;
        const int n = in.npml[a][s];
        if (i < 1 || i > n) return;
        const double nm1 = (double)n - 1.0;
        {  // E depth i = 1..n (ref :3404-3450 restated in FP64)
            const double g = (double)(n - i) / nm1;
            const double sg = in.sig_max[a] * gpow(g, in.m);
            const double al = in.alpha_max * (((double)i - 1.0) / nm1);
            const double ka = 1.0 + (in.kappa_max - 1.0) * gpow(g, in.m);
            const double b = exp(-((sg / ka + al) * dt / kEp0d));
            const double cc = (sg == 0.0 && al == 0.0 && i == n) ? 0.0 : sg * (b - 1.0) / (sg + ka * al) / ka;
            cp_row(cpml, a, s, 0)[i] = (float)b;
            cp_row(cpml, a, s, 1)[i] = (float)cc;
            cp_row(cpml, a, s, 2)[i] = (float)ka;
        }
        if (i <= n - 1) {  // H depth i = 1..n-1, half a cell in
            const double g = ((double)(n - i) - 0.5) / nm1;
            const double sg = in.sig_max[a] * gpow(g, in.m);
            const double al = in.alpha_max * (((double)i - 0.5) / nm1);
            const double ka = 1.0 + (in.kappa_max - 1.0) * gpow(g, in.m);
            const double b = exp(-((sg / ka + al) * dt / kEp0d));
            const double cc = sg * (b - 1.0) / (sg + ka * al) / ka;
            cp_row(cpml, a, s, 3)[i] = (float)b;
            cp_row(cpml, a, s, 4)[i] = (float)cc;
            cp_row(cpml, a, s, 5)[i] = (float)ka;
        }
        return;
    }
    u -= 3 * 2 * CP_STRIDE;
    // den tables, ref :3584-3666: 1 / (kappa d) in the slabs, 1 / d elsewhere
    for (int a = 0; a < 3; a++) {
        const int Na = in.N[a];
        if (u < Na - 1) {
            const int i = u + 1, n1 = in.npml[a][0], n2 = in.npml[a][1];
            auto kap = [&](int side, int q, bool e_tab) {
                const double nm1 = (double)in.npml[a][side] - 1.0;
                const double g = e_tab ? (double)(in.npml[a][side] - q) / nm1 : ((double)(in.npml[a][side] - q) - 0.5) / nm1;
                return 1.0 + (in.kappa_max - 1.0) * gpow(g, in.m);
            };
            double vh, ve;
            if (i <= n1 - 1) vh = 1.0 / (kap(0, i, false) * in.dl[a]);
            else if (i >= Na + 1 - n2) vh = 1.0 / (kap(1, Na - i, false) * in.dl[a]);
            else vh = 1.0 / in.dl[a];
            if (i <= n1) ve = 1.0 / (kap(0, i, true) * in.dl[a]);
            else if (i >= Na + 1 - n2) ve = 1.0 / (kap(1, Na + 1 - i, true) * in.dl[a]);
            else ve = 1.0 / in.dl[a];
            den[in.den_off[a] + i - 1] = (float)vh;
            den[in.den_off[a] + (Na + 1) + i - 1] = (float)ve;
            return;
        }
        u -= Na - 1;
    }
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e) + " (" + what + ")");
    }
}

}  // namespace

void coef_tables_fp64(HostModel& m) {
    const Deck& d = m.d;
    CoefIn in{};
    in.nmat = (int)m.mats.size();
    in.npoles = m.npoles;
    in.m = d.cpml_m;
    in.dt = (double)d.del_t;
    const int N[3] = {d.X, d.Y, d.Z};
    const float dl[3] = {d.dx, d.dy, d.dz};
    for (int a = 0; a < 3; a++) {
        in.N[a] = N[a];
        in.dl[a] = (double)dl[a];
        in.sig_max[a] = (double)d.sig_max[a];
        for (int s = 0; s < 2; s++) in.npml[a][s] = d.npml[a][s];
    }
    in.alpha_max = (double)d.alpha_max;
    in.kappa_max = (double)d.kappa_max;
    const size_t cp_n = (size_t)3 * 2 * 6 * CP_STRIDE;
    size_t den_n = 0;
    for (int a = 0; a < 3; a++) {
        in.den_off[a] = (long long)den_n;
        den_n += (size_t)2 * (N[a] + 1);
    }
    AemMaterial* dm = nullptr;
    AemUniformCoef* du = nullptr;
    float *dc = nullptr, *dd = nullptr;
    std::vector<float> cp(cp_n), den(den_n);
    try {
        check(cudaMalloc(&dm, m.mats.size() * sizeof(AemMaterial)), "coefficient tables");
        check(cudaMalloc(&du, m.ucoef.size() * sizeof(AemUniformCoef)), "coefficient tables");
        check(cudaMalloc(&dc, cp_n * sizeof(float)), "coefficient tables");
        check(cudaMalloc(&dd, den_n * sizeof(float)), "coefficient tables");
        check(cudaMemcpy(dm, m.mats.data(), m.mats.size() * sizeof(AemMaterial), cudaMemcpyHostToDevice), "upload");
        check(cudaMemcpy(du, m.ucoef.data(), m.ucoef.size() * sizeof(AemUniformCoef), cudaMemcpyHostToDevice), "upload");
        check(cudaMemset(dc, 0, cp_n * sizeof(float)), "clear");
        check(cudaMemset(dd, 0, den_n * sizeof(float)), "clear");
        const long long work = (long long)in.nmat * 3 + 3 * 2 * CP_STRIDE + (N[0] + N[1] + N[2]);
        k_coef_fp64<<<(unsigned)((work + 127) / 128), 128>>>(dm, in, du, dc, dd);
        check(cudaGetLastError(), "k_coef_fp64");
        check(cudaMemcpy(m.ucoef.data(), du, m.ucoef.size() * sizeof(AemUniformCoef), cudaMemcpyDeviceToHost), "download");
        check(cudaMemcpy(cp.data(), dc, cp_n * sizeof(float), cudaMemcpyDeviceToHost), "download");
        check(cudaMemcpy(den.data(), dd, den_n * sizeof(float), cudaMemcpyDeviceToHost), "download");
    } catch (...) {
        cudaFree(dm); cudaFree(du); cudaFree(dc); cudaFree(dd);
        throw;
    }
    cudaFree(dm); cudaFree(du); cudaFree(dc); cudaFree(dd);
    auto row = [&](int a, int s, int which) { return &cp[(((size_t)a * 2 + s) * 6 + which) * CP_STRIDE]; };
    size_t off = 0;
    for (int a = 0; a < 3; a++) {
        for (int s = 0; s < 2; s++) {
            const int n = d.npml[a][s];
            for (int i = 1; i <= n; i++) {
                m.be[a][s][i - 1] = row(a, s, 0)[i];
                m.ce[a][s][i - 1] = row(a, s, 1)[i];
            }
            for (int i = 1; i <= n - 1; i++) {
                m.bh[a][s][i - 1] = row(a, s, 3)[i];
                m.ch[a][s][i - 1] = row(a, s, 4)[i];
            }
        }
        for (int i = 1; i <= N[a] - 1; i++) {
            m.den_h[a][i - 1] = den[off + i - 1];
            m.den_e[a][i - 1] = den[off + (N[a] + 1) + i - 1];
        }
        off += (size_t)2 * (N[a] + 1);
    }
}

}  // namespace aem
