// aem_finalize.cu -- post-loop processing and output files of a run,
// main_fdtd/fdtd_solver.f90:8338-8807.
//
// The .dat file keeps the reference's line numbers and whitespace token
// columns (what utility_scripts/post_processor*.py parse); numbers use one
// fixed format (reals "%.9E", integers "%12d").
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "aem_dev.cuh"
#include "aem_model.h"
#include "aem_solver.h"

namespace aem {

#define AEM_CUDA(x)                                                                                     \
    do {                                                                                                \
        cudaError_t e_ = (x);                                                                           \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + \
                                                        " at " #x);                                     \
    } while (0)

namespace {

using cplx = std::complex<float>;

// Far-field rE_theta / rE_phi of one angle from its six binned components
// (W x,y,z then U x,y,z), ref :8483-8534, in the host expression's FP32
// operation order: Wt = (wx c1) c2 + (wy c1) s2 - wz s1, Wp = (-1 wx) s2 +
// wy c2 (U likewise), Et = (-1 eta) Wt - Up, Ep = (-1 eta) Wp + Ut.  The
// angle's cosines and sines come from the host.
// The accumulators are FP64 (rounded to FP32 here, the precision the
// reference's U/W arrays hold); a constant-k run's real and imaginary
// planes are first joined into complex64 (k_ff_join).
__device__ inline float to_v(double x, float) { return (float)x; }
__device__ inline cf to_v(cf x, cf) { return x; }
template <typename V, typename A>
__device__ inline void ff_pol(const A* uw, long long stride, long long j, const float* cs, float eta, V& Et, V& Ep) {
    const float c1 = cs[0], s1 = cs[1], c2 = cs[2], s2 = cs[3];
    const V z{};
    const V wx = to_v(uw[j], z), wy = to_v(uw[stride + j], z), wz = to_v(uw[2 * stride + j], z);
    const V ux = to_v(uw[3 * stride + j], z), uy = to_v(uw[4 * stride + j], z), uz = to_v(uw[5 * stride + j], z);
    const V Wt = wx * c1 * c2 + wy * c1 * s2 - wz * s1;
    const V Wp = -1.0f * wx * s2 + wy * c2;
    const V Ut = ux * c1 * c2 + uy * c1 * s2 - uz * s1;
    const V Up = -1.0f * ux * s2 + uy * c2;
    const float me = -1.0f * eta;
    Et = me * Wt - Up;
    Ep = me * Wp + Ut;
}
// the real and imaginary FP64 planes of a constant-k run -> complex64
__global__ void k_ff_join(const double* re, const double* im, cf* out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = cf{(float)re[i], (float)im[i]};
}

__device__ inline bool nz(float v) { return v != 0.0f; }
__device__ inline bool nz(cf v) { return v.x != 0.0f || v.y != 0.0f; }

// One CTA per angle: the first bins (1-based) where Ep and Et are non-zero
// give the output window start o (ref :8520-8530), then the T values from o
// are written.  UW rows: [component][angle][L]; an angle whose delays equal
// an earlier one's reads that angle's rows (canon).
template <typename V, typename A>
__global__ void k_ff_out(const A* UW, int nff, long long L, int len_ff, int T, const float* trig, float eta,
                         const int* canon, V* eth, V* eph, int* out_time) {
    const int i = blockIdx.x;
    const A* uw = UW + (long long)canon[i] * L;
    const long long stride = (long long)nff * L;
    const float* cs = trig + 4 * i;
    __shared__ int first[2];
    if (threadIdx.x == 0) first[0] = first[1] = len_ff;
    __syncthreads();
    int dp = len_ff, dt = len_ff;
    for (int j = 1 + threadIdx.x; j <= len_ff; j += blockDim.x) {
        if (j >= dp && j >= dt) break;
        V Et, Ep;
        ff_pol(uw, stride, j - 1, cs, eta, Et, Ep);
        if (nz(Ep) && j < dp) dp = j;
        if (nz(Et) && j < dt) dt = j;
    }
    atomicMin(&first[0], dp);
    atomicMin(&first[1], dt);
    __syncthreads();
    int o = min(first[0], first[1]);
    if (o > len_ff - T + 1) o = len_ff - T + 1;
    if (threadIdx.x == 0) out_time[i] = o;
    for (int j = 1 + threadIdx.x; j <= T; j += blockDim.x) {
        V Et, Ep;
        const long long b = (long long)j + o - 2;  // 0-based bin
        if (b < 0 || b >= len_ff) {                // only when len_ff < T
            eth[(long long)i * T + j - 1] = V();
            eph[(long long)i * T + j - 1] = V();
            continue;
        }
        ff_pol(uw, stride, b, cs, eta, Et, Ep);
        eth[(long long)i * T + j - 1] = Et;
        eph[(long long)i * T + j - 1] = Ep;
    }
}

// device buffer -> host, complex or real
std::vector<cplx> fetch(const void* dev, size_t n, bool kmax, cudaStream_t s, size_t& counter) {
    std::vector<cplx> out(n);
    if (!n) return out;
    counter += n * (kmax ? sizeof(cplx) : sizeof(float));
    if (kmax) {
        AEM_CUDA(cudaMemcpyAsync(out.data(), dev, n * sizeof(cplx), cudaMemcpyDeviceToHost, s));
        AEM_CUDA(cudaStreamSynchronize(s));
    } else {
        std::vector<float> t(n);
        AEM_CUDA(cudaMemcpyAsync(t.data(), dev, n * sizeof(float), cudaMemcpyDeviceToHost, s));
        AEM_CUDA(cudaStreamSynchronize(s));
        for (size_t q = 0; q < n; q++) out[q] = cplx(t[q], 0.0f);
    }
    return out;
}

void wreal(FILE* f, double v) { std::fprintf(f, "  %.9E", v); }
void wline(FILE* f, cplx v, bool kmax) {
    wreal(f, v.real());
    if (kmax) wreal(f, v.imag());
    std::fputc('\n', f);
}

}  // namespace

void Solver::finalize_and_write() {
    const Deck& d = m_.d;
    const bool K = d.kmax;
    const int T = d.steps;
    flush_farfield(done_);
    flush_farfield_tail();
    full_flush();
    AEM_CUDA(cudaStreamSynchronize(stream_));
    const float mu0 = 1.25663706E-6f, ep0 = 8.85418782E-12f, c0 = 299792458.0f, pi = 3.14159265358979323846f;
    if (FF_.err) {
        int err = 0;
        AEM_CUDA(cudaMemcpy(&err, FF_.err, sizeof err, cudaMemcpyDeviceToHost));
        d2h_bytes_ += sizeof err;
        if (err) throw std::runtime_error("far-field binning: " + std::to_string(err) + " contributions outside their window");
    }
    if (P_.err) {
        int err = 0;
        AEM_CUDA(cudaMemcpy(&err, P_.err, sizeof err, cudaMemcpyDeviceToHost));
        d2h_bytes_ += sizeof err;
        if (err) throw std::runtime_error("fused field update: " + std::to_string(err) + " tiles gave up waiting for their copies");
    }

    // plane sums, normalised per ref :8342-8361 / :8412-8435
    std::vector<cplx> refl, trans, refl_tm, trans_tm;
    if (TP_.plane_sum) {
        refl = fetch(TP_.refl, T, K, stream_, d2h_bytes_);
        trans = fetch(TP_.trans, T, K, stream_, d2h_bytes_);
        if (K) { refl_tm = fetch(TP_.refl_tm, T, K, stream_, d2h_bytes_); trans_tm = fetch(TP_.trans_tm, T, K, stream_, d2h_bytes_); }
        const int a = TP_.axis, b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
        const int N[3] = {d.X, d.Y, d.Z};
        // the reference multiplies the two transverse (size-2.0) factors in the
        // order (y,z) / (x,z) / (y,x)
        float den = a == 2 ? ((float)N[1] - 2.0f) * ((float)N[0] - 2.0f) : ((float)N[b] - 2.0f) * ((float)N[c] - 2.0f);
        for (int n = 0; n < T; n++) {
            refl[n] = refl[n] / den;
            trans[n] = trans[n] / den;
            if (K) { refl_tm[n] = refl_tm[n] / den; trans_tm[n] = trans_tm[n] / den; }
        }
    }
    // incident waveform, ref :8366-8408 (standard) / :8438-8479 (kmax)
    std::vector<cplx> inc(T, cplx(0, 0));
    auto eorv = [&](float amp, float tc, float posd) -> cplx {
        float a = (d.t_spread - ((tc - 1.0f) * d.del_t) - 1.0f / c0 * posd) / d.spread;
        if (!K) {
            if (d.pulse_type == 1) return cplx(amp * std::exp(-0.5f * (a * a)), 0);
            if (d.pulse_type == 2) return cplx(amp * -1.0f * a * std::exp(0.5f) * std::exp(-0.5f * (a * a)), 0);
            return cplx(0, 0);
        }
        float env = amp * std::exp(-0.5f * (a * a));
        float ph = 2.0f * pi * d.f_adj * ((tc - 1.0f) * d.del_t - 1.0f / c0 * posd);
        return env * cplx(std::cos(ph), std::sin(ph));
    };
    if (d.pw_amp > 0)
        for (int n = 1; n <= T; n++) inc[n - 1] = eorv(d.pw_amp, (float)n, 0.0f * d.dx);
    if (d.ant_amp > 0 && d.exc_port >= 1 && d.exc_port <= (int)d.ports.size()) {
        // matched 1-D line driven alone (the "clear" incident voltage)
        const Port& p = d.ports[d.exc_port - 1];
        const float dl[3] = {d.dx, d.dy, d.dz};
        const float st = dl[p.dir];
        const int Pn = d.port_array_size;
        std::vector<cplx> V(2 * Pn + 1, cplx(0, 0)), C(2 * Pn + 1, cplx(0, 0));  // 1-based, C[0] = 0
        const float cI = (1.0f / p.L) * (d.del_t / st), cV = (1.0f / p.C) * (d.del_t / st);
        const float cS = (1.0f / std::sqrt(p.C * p.L)) * (d.del_t / st);
        for (int n = 1; n <= T; n++) {
            for (int j = 1; j <= 2 * Pn - 1; j++) C[j] = C[j] - cI * (V[j + 1] - V[j]);
            C[Pn] = C[Pn] - cI * eorv(d.ant_amp, (float)n, 0.0f * st);
            for (int j = 1; j <= 2 * Pn - 1; j++) V[j] = V[j] - cV * (C[j] - C[j - 1]);
            V[Pn] = V[Pn] + cS * eorv(d.ant_amp, (float)n + 0.5f, 0.5f * st);
            inc[n - 1] = V[Pn];
        }
    }
    // far field, ref :8483-8534
    const int nff = d.n_ff;
    std::vector<std::vector<cplx>> eth(nff), eph(nff);
    data_out_time.assign(nff, 1);
    if (nff > 0) {
        // the transform runs on the device; only each angle's T-step window
        // comes back
        const size_t L = FF_.len;
        const float eta = std::sqrt(mu0 / ep0);
        std::vector<float> trig(4 * (size_t)nff);
        for (int i = 0; i < nff; i++) {
            const float a1 = d.ff_theta[i], a2 = d.ff_phi[i];
            trig[4 * i] = std::cos(a1); trig[4 * i + 1] = std::sin(a1);
            trig[4 * i + 2] = std::cos(a2); trig[4 * i + 3] = std::sin(a2);
        }
        std::vector<int> canon(nff);
        for (int i = 0; i < nff; i++) canon[i] = i < (int)ff_canon_.size() ? ff_canon_[i] : i;
        float* d_trig = (float*)alloc(trig.size() * sizeof(float));
        int* d_canon = (int*)alloc(canon.size() * sizeof(int));
        int* d_time = (int*)alloc(canon.size() * sizeof(int));
        void* d_eth = alloc((size_t)nff * T * es_);
        void* d_eph = alloc((size_t)nff * T * es_);
        AEM_CUDA(cudaMemcpyAsync(d_trig, trig.data(), trig.size() * sizeof(float), cudaMemcpyHostToDevice, stream_));
        AEM_CUDA(cudaMemcpyAsync(d_canon, canon.data(), canon.size() * sizeof(int), cudaMemcpyHostToDevice, stream_));
        if (K) {
            const long long nuw = (long long)6 * nff * L;
            cf* d_uw = (cf*)alloc((size_t)nuw * sizeof(cf));
            const double* uw = (const double*)FF_.UW;
            k_ff_join<<<(unsigned)std::min<long long>((nuw + 255) / 256, 148 * 8), 256, 0, stream_>>>(uw, uw + nuw, d_uw, nuw);
            k_ff_out<cf, cf><<<nff, 256, 0, stream_>>>(d_uw, nff, (long long)L, d.len_ff, T, d_trig, eta, d_canon,
                                                       (cf*)d_eth, (cf*)d_eph, d_time);
        } else
            k_ff_out<float, double><<<nff, 256, 0, stream_>>>((const double*)FF_.UW, nff, (long long)L, d.len_ff, T, d_trig,
                                                              eta, d_canon, (float*)d_eth, (float*)d_eph, d_time);
        AEM_CUDA(cudaGetLastError());
        AEM_CUDA(cudaMemcpyAsync(data_out_time.data(), d_time, nff * sizeof(int), cudaMemcpyDeviceToHost, stream_));
        d2h_bytes_ += nff * sizeof(int);
        std::vector<cplx> th = fetch(d_eth, (size_t)nff * T, K, stream_, d2h_bytes_);
        std::vector<cplx> ph = fetch(d_eph, (size_t)nff * T, K, stream_, d2h_bytes_);
        for (int i = 0; i < nff; i++) {
            eth[i].assign(th.begin() + (size_t)i * T, th.begin() + (size_t)(i + 1) * T);
            eph[i].assign(ph.begin() + (size_t)i * T, ph.begin() + (size_t)(i + 1) * T);
        }
    }
    std::vector<std::vector<cplx>> vout(d.ports.size());
    for (size_t q = 0; q < d.ports.size(); q++) vout[q] = fetch(PS_.p[q].vout, T, K, stream_, d2h_bytes_);
    std::vector<cplx> pc[3];
    if (TP_.ff_pc)
        for (int c = 0; c < 3; c++) pc[c] = fetch(TP_.pc[c], T, K, stream_, d2h_bytes_);

    // keep host copies for callers of the library
    auto split = [](const std::vector<cplx>& v, std::vector<double>& re, std::vector<double>& im) {
        re.resize(v.size()); im.resize(v.size());
        for (size_t q = 0; q < v.size(); q++) { re[q] = v[q].real(); im[q] = v[q].imag(); }
    };
    split(inc, incident_re, incident_im);
    split(refl, refl_re, refl_im); split(trans, trans_re, trans_im);
    split(refl_tm, refl_tm_re, refl_tm_im); split(trans_tm, trans_tm_re, trans_tm_im);
    vout_re.assign(vout.size(), {}); vout_im.assign(vout.size(), {});
    for (size_t q = 0; q < vout.size(); q++) split(vout[q], vout_re[q], vout_im[q]);
    eth_re.assign(nff, {}); eth_im.assign(nff, {}); eph_re.assign(nff, {}); eph_im.assign(nff, {});
    for (int i = 0; i < nff; i++) { split(eth[i], eth_re[i], eth_im[i]); split(eph[i], eph_re[i], eph_im[i]); }
    for (int c = 0; c < 3; c++) split(pc[c], pc_re[c], pc_im[c]);

    // ---- <name>.dat, ref :8538-8645 (standard) / :8649-8784 (kmax)
    std::string path = outdir_.empty() ? d.filename : outdir_ + "/" + d.filename;
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::fprintf(f, " x steps = %12d\n", d.X - 1 - d.pbc[0]);
    std::fprintf(f, " y steps = %12d\n", d.Y - 1 - d.pbc[1]);
    std::fprintf(f, " z steps = %12d\n", d.Z - 1 - d.pbc[2]);
    std::fprintf(f, " delta x,y,z = "); wreal(f, d.dx); wreal(f, d.dy); wreal(f, d.dz); std::fputc('\n', f);
    std::fprintf(f, " time step = "); wreal(f, d.del_t); std::fputc('\n', f);
    std::fprintf(f, " number of time steps = %12d\n", d.steps);
    if (!K) { std::fprintf(f, " minimum time steps needed (but more recommended) = "); wreal(f, d.min_steps); std::fputc('\n', f); }
    else std::fprintf(f, " minimum time steps needed N/A\n");
    if (!K) { std::fprintf(f, " freq parameter = "); wreal(f, d.f_center); std::fputc('\n', f); std::fprintf(f, " pulse type = %12d\n", d.pulse_type); }
    else { std::fprintf(f, " freq center = "); wreal(f, d.f_center); std::fputc('\n', f); std::fprintf(f, " pulse type = N/A\n"); }
    std::fprintf(f, " slice = %12d\n", d.slice_dir);
    std::fprintf(f, " slice location = %12d\n", d.slice_loc);
    std::fprintf(f, " video size_a = %12d\n", d.vid1);
    std::fprintf(f, " video size_b = %12d\n", d.vid2);
    std::fprintf(f, " number of far field angles = %12d\n", nff);
    std::fprintf(f, " number of internal ports = %12d\n", (int)d.ports.size());
    std::fprintf(f, " number of spice ports = %12d\n", 0);
    if (!K) std::fprintf(f, " simulation type%12d%12d%12d\n", d.pbc[0], d.pbc[1], d.pbc[2]);
    else {
        std::fprintf(f, " simulation type%12d%12d%12d%12d\n", d.pbc[0], d.pbc[1], d.pbc[2], d.k_direction);
        std::fprintf(f, " simulation is k vector method w/ k1,k2:\n");
        if (d.pbc[1] + d.pbc[2] == 2) { wreal(f, d.kc[1]); wreal(f, d.kc[2]); }
        else if (d.pbc[0] + d.pbc[2] == 2) { wreal(f, d.kc[0]); wreal(f, d.kc[2]); }
        else if (d.pbc[0] + d.pbc[1] == 2) { wreal(f, d.kc[0]); wreal(f, d.kc[1]); }
        std::fputc('\n', f);
        std::fprintf(f, " mode type is 0 for TE and 1 for TM:%12d\n", d.mode_type);
    }
    if (d.excitation == "plane wave")
        std::fprintf(f, K ? " incident E-field wave: (not used in post processor bc r(k))\n" : " incident E-field wave:\n");
    if (d.excitation == "antenna") std::fprintf(f, " incident voltage wave at port %12d\n", d.exc_port);
    for (int n = 0; n < T; n++) wline(f, inc[n], K);
    if (!K) {
        if (d.pbc[0] + d.pbc[1] + d.pbc[2] == 2 && d.excitation == "plane wave") {
            bool direct = (d.pbc[0] == 0 && d.phi == 0) || (d.pbc[1] == 0 && (d.phi > 89.0f * pi / 180.0f && d.phi < 91.0f * pi / 180.0f)) ||
                          (d.pbc[2] == 0 && d.theta == 0);
            std::fprintf(f, " reflected wave for PBC:\n");
            for (int n = 0; n < T; n++) wline(f, direct ? refl[n] : trans[n], K);
            std::fprintf(f, " transmitted wave for PBC:\n");
            for (int n = 0; n < T; n++) wline(f, direct ? trans[n] : refl[n], K);
        }
    } else {
        const std::vector<cplx>* blk[4];
        if (d.k_direction == 1) { blk[0] = &refl; blk[1] = &refl_tm; blk[2] = &trans; blk[3] = &trans_tm; }
        else { blk[0] = &trans; blk[1] = &trans_tm; blk[2] = &refl; blk[3] = &refl_tm; }
        const char* hd[4] = {" TE Refl Wave:", " TM Refl Wave:", " TE Trans Wave:", " TM Trans Wave:"};
        for (int b = 0; b < 4; b++) {
            std::fprintf(f, "%s\n", hd[b]);
            for (int n = 0; n < T; n++) wline(f, blk[b]->empty() ? cplx(0, 0) : (*blk[b])[n], K);
        }
    }
    for (int i = 0; i < nff; i++) {
        float t_ = 180.0f / pi * d.ff_theta[i], p_ = 180.0f / pi * d.ff_phi[i];
        std::fprintf(f, " far field rE theta polarization at theta,phi:\n"); wreal(f, t_); wreal(f, p_); std::fputc('\n', f);
        for (int j = 0; j < T; j++) wline(f, eth[i][j], K);
        std::fprintf(f, " far field rE phi polarization at theta,phi:\n"); wreal(f, t_); wreal(f, p_); std::fputc('\n', f);
        for (int j = 0; j < T; j++) wline(f, eph[i][j], K);
    }
    for (size_t q = 0; q < d.ports.size(); q++) {
        std::fprintf(f, " recieved voltage at port %12d w/ Z\n", (int)q + 1);
        wreal(f, std::sqrt(d.ports[q].L / d.ports[q].C)); std::fputc('\n', f);
        for (int j = 0; j < T; j++) wline(f, vout[q][j], K);
    }
    if (nff > 0) {
        std::fprintf(f, " far field phase correction time information:\n");
        for (int i = 0; i < nff; i++) { wreal(f, (d.r_relay / c0) - (float)(data_out_time[i] - 1) * d.del_t); std::fputc('\n', f); }
    }
    if (nff > 0 && d.pw_amp > 0) {
        if (!K) {
            std::fprintf(f, " incident for far field phase centering:\n");
            const float w0 = (std::cos(d.pol) * std::sin(d.phi) - std::sin(d.pol) * std::cos(d.theta) * std::cos(d.phi));
            const float w1 = (-1.0f * std::cos(d.pol) * std::cos(d.phi) - std::sin(d.pol) * std::cos(d.theta) * std::sin(d.phi));
            const float w2 = (std::sin(d.pol) * std::sin(d.theta));
            for (int n = 0; n < T; n++) wline(f, pc[0][n] * w0 + pc[1][n] * w1 + pc[2][n] * w2, K);
        } else {
            std::fprintf(f, " incident for far field phase centering (Ex,Ey,Ez):\n");
            for (int c = 0; c < 3; c++)
                for (int n = 0; n < T; n++) wline(f, pc[c][n], K);
        }
    }
    std::fclose(f);

    // point probes (extension `probe i j k`): <name>_probes.dat, a header
    // line per probe component followed by its T samples, in the .dat
    // file's number format; the reference has no point probes
    if (TP_.nprobe > 0) {
        std::vector<cplx> pv = fetch(TP_.prb, (size_t)3 * TP_.nprobe * T, K, stream_, d2h_bytes_);
        const std::string base = d.filename.substr(0, d.filename.size() >= 4 ? d.filename.size() - 4 : 0);
        const std::string fn = (outdir_.empty() ? "" : outdir_ + "/") + base + "_probes.dat";
        FILE* pf = std::fopen(fn.c_str(), "w");
        if (!pf) throw std::runtime_error("cannot write " + fn);
        std::fprintf(pf, " number of point probes = %12d\n", TP_.nprobe);
        static const char* cn[3] = {"Ex", "Ey", "Ez"};
        for (int q = 0; q < TP_.nprobe; q++)
            for (int c = 0; c < 3; c++) {
                std::fprintf(pf, " point probe %12d %s at cell%12d%12d%12d\n", q + 1, cn[c], TP_.prb_idx[q][0],
                             TP_.prb_idx[q][1], TP_.prb_idx[q][2]);
                for (int n = 0; n < T; n++) wline(pf, pv[((size_t)q * 3 + c) * T + n], K);
            }
        std::fclose(pf);
    }

    // video slices, one Fortran unformatted record per file, ref :8788-8807
    if (TP_.video) {
        const char* nm[6] = {"Ex", "Hx", "Ey", "Hy", "Ez", "Hz"};
        const size_t n = (size_t)TP_.v1 * TP_.v2 * T;
        for (int q = 0; q < 6; q++) {
            std::vector<cplx> v = fetch(TP_.vid[q], n, K, stream_, d2h_bytes_);
            std::string base = d.filename.substr(0, d.filename.size() >= 4 ? d.filename.size() - 4 : 0);
            std::string fn = (outdir_.empty() ? "" : outdir_ + "/") + base + "_video_" + nm[q] + ".bin";
            FILE* vf = std::fopen(fn.c_str(), "wb");
            if (!vf) continue;
            int32_t Lr = (int32_t)(n * 4 * (K ? 2 : 1));
            std::fwrite(&Lr, 4, 1, vf);
            for (size_t e = 0; e < n; e++) {
                float re = v[e].real(), im = v[e].imag();
                std::fwrite(&re, 4, 1, vf);
                if (K) std::fwrite(&im, 4, 1, vf);
            }
            std::fwrite(&Lr, 4, 1, vf);
            std::fclose(vf);
        }
    }
}

// final field component in the reference's own array layout; comp 6 gives
// the per-cell material indices the run uses (0 = vacuum, r = r-th volume
// material of the deck)
void Solver::get_field(int comp, std::vector<double>& re, std::vector<double>& im, int dims[3]) {
    const Deck& d = m_.d;
    const int X = d.X, Y = d.Y, Z = d.Z;
    if (comp == 6) {  // the cells' material indices, cells 1..N-1 (not a periodic axis' duplicate)
        for (int a = 0; a < 3; a++) dims[a] = (a == 0 ? X : a == 1 ? Y : Z) - 1 - d.pbc[a];
        std::vector<uint8_t> ids((size_t)m_.cells);
        AEM_CUDA(cudaMemcpyAsync(ids.data(), P_.cell, ids.size(), cudaMemcpyDeviceToHost, stream_));
        AEM_CUDA(cudaStreamSynchronize(stream_));
        d2h_bytes_ += ids.size();
        re.assign((size_t)dims[0] * dims[1] * dims[2], 0.0);
        im.assign(re.size(), 0.0);
        for (int k = 1; k <= dims[2]; k++)
            for (int j = 1; j <= dims[1]; j++)
                for (int i = 1; i <= dims[0]; i++)
                    re[((size_t)(k - 1) * dims[1] + (j - 1)) * dims[0] + (i - 1)] = ids[m_.lin(i, j, k)];
        return;
    }
    static const int ext[6][3] = {{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {0, -1, -1}, {-1, 0, -1}, {-1, -1, 0}};
    dims[0] = X + ext[comp][0]; dims[1] = Y + ext[comp][1]; dims[2] = Z + ext[comp][2];
    std::vector<cplx> all = fetch(comp < 3 ? P_.E[comp] : P_.H[comp - 3], (size_t)m_.cells, d.kmax, stream_, d2h_bytes_);
    size_t n = (size_t)dims[0] * dims[1] * dims[2];
    re.assign(n, 0.0); im.assign(n, 0.0);
    const int N[3] = {X, Y, Z};
    for (int k = 1; k <= dims[2]; k++)
        for (int j = 1; j <= dims[1]; j++)
            for (int i = 1; i <= dims[0]; i++) {
                const int idx[3] = {i, j, k};
                bool ok = true;
                cplx ph(1, 0);
                for (int a = 0; a < 3; a++) {
                    if (!d.pbc[a]) { if (idx[a] > m_.S[a]) ok = false; continue; }
                    // reference index N-1 duplicates index 1 (times the Bloch phase)
                    if (idx[a] == N[a] - 1) {
                        const float dl[3] = {d.dx, d.dy, d.dz};
                        float th = d.kc[a] * (float)(N[a] - 2) * dl[a];
                        ph *= cplx(std::cos(th), -std::sin(th));
                    }
                    if (idx[a] > N[a] - 1) ok = false;
                }
                if (!ok) continue;
                cplx v = all[m_.lin(i, j, k)] * ph;
                size_t o = ((size_t)(k - 1) * dims[1] + (j - 1)) * dims[0] + (i - 1);
                re[o] = v.real(); im[o] = v.imag();
            }
}

}  // namespace aem
