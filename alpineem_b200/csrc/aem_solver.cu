// aem_solver.cu -- device state and time loop of one run.
//
// The time loop order follows main_fdtd/fdtd_solver.f90:4440-8299:
//   H update (+sheets, TF/SF, CPML, PBC)  -> port H half-step
//   E update (+sheets, Drude, TF/SF, CPML, PBC) -> port E half-step
//   far-field currents and binning, plane sums, phase-centre, video.
#include "aem_solver.h"

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <stdexcept>

namespace aem {

#define AEM_CUDA(x)                                                                                     \
    do {                                                                                                \
        cudaError_t e_ = (x);                                                                           \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + \
                                                        " at " #x);                                     \
    } while (0)

static std::string dir_of(const std::string& p) {
    size_t s = p.find_last_of('/');
    return s == std::string::npos ? std::string() : p.substr(0, s);
}

void* Solver::alloc(size_t bytes) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();  // do not leave the failure pending for later calls
        throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e) + " allocating " +
                                 std::to_string(bytes) + " bytes");
    }
    AEM_CUDA(cudaMemsetAsync(p, 0, bytes, stream_));
    bufs_.push_back(p);
    dev_bytes_ += bytes;
    return p;
}

template <typename V>
void* Solver::upload(const std::vector<V>& v) {
    void* p = alloc(v.size() * sizeof(V));
    if (!v.empty()) AEM_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice, stream_));
    return p;
}

Solver::Solver(const std::string& inputs_path, bool kmax, const std::string& outdir) : outdir_(outdir) {
    AEM_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    m_.d = parse_deck_file(inputs_path, kmax);
    derive(m_.d);
    build_model(m_, dir_of(inputs_path));
    es_ = kmax ? 8 : 4;
    setup_params();
    setup_ports();
    setup_farfield();
    setup_taps();
    AEM_CUDA(cudaStreamSynchronize(stream_));
}

Solver::~Solver() {
    if (stream_) cudaStreamSynchronize(stream_);
    for (void* p : bufs_) cudaFree(p);
    if (stream_) cudaStreamDestroy(stream_);
}

long long Solver::cell_count() const {
    const Deck& d = m_.d;
    return (long long)(d.X - 1) * (d.Y - 1) * (d.Z - 1);
}

// 49 B per cell-update (6 FP32 components read + written, 1 B material ID)
// plus 32 B per CPML slab a cell belongs to (2 E-psi + 2 H-psi read and
// written); complex fields double the field and psi terms.
double Solver::algorithmic_bytes_per_step() const {
    const Deck& d = m_.d;
    const double fe = es_;
    double cells = (double)cell_count();
    double slab = 0;
    const int N[3] = {d.X, d.Y, d.Z};
    for (int a = 0; a < 3; a++) {
        int depth = (d.npml[a][0] > 0 ? d.npml[a][0] - 1 : 0) + (d.npml[a][1] > 0 ? d.npml[a][1] - 1 : 0);
        double face = 1;
        for (int b = 0; b < 3; b++) if (b != a) face *= (double)(N[b] - 1);
        slab += depth * face;
    }
    return cells * (12.0 * fe + 1.0) + slab * 8.0 * fe;
}

void Solver::setup_params() {
    const Deck& d = m_.d;
    AemParams& P = P_;
    std::memset(&P, 0, sizeof P);
    P.X = d.X; P.Y = d.Y; P.Z = d.Z;
    for (int a = 0; a < 3; a++) P.per[a] = d.pbc[a];
    P.SX = m_.S[0]; P.SY = m_.S[1]; P.SZ = m_.S[2];
    P.PX = m_.PX;
    P.plane = m_.plane;
    P.kmax = d.kmax ? 1 : 0;
    const float dl[3] = {d.dx, d.dy, d.dz};
    const int N[3] = {d.X, d.Y, d.Z};
    for (int a = 0; a < 3; a++) {
        // exp(+i k (N-2) d), ref :6686
        float th = d.kc[a] * (float)(N[a] - 2) * dl[a];
        P.bloch_re[a] = std::cos(th);
        P.bloch_im[a] = std::sin(th);
        P.del[a] = dl[a];
    }
    const float mu0 = 1.25663706E-6f, ep0 = 8.85418782E-12f, c0 = 299792458.0f, pi = 3.14159265358979323846f;
    P.DB = d.del_t / mu0;
    P.dt = d.del_t;
    for (int c = 0; c < 3; c++) {
        P.E[c] = alloc((size_t)m_.cells * es_);
        P.H[c] = alloc((size_t)m_.cells * es_);
    }
    P.cell = (const uint8_t*)upload(m_.cell_id);
    for (int a = 0; a < 3; a++) {
        P.npml[a][0] = d.npml[a][0];
        P.npml[a][1] = d.npml[a][1];
        P.den_e[a] = (const float*)upload(m_.den_e[a]);
        P.den_h[a] = (const float*)upload(m_.den_h[a]);
        for (int s = 0; s < 2; s++)
            for (int q = 0; q < AEM_MAX_PML; q++) {
                P.be[a][s][q] = m_.be[a][s][q]; P.ce[a][s][q] = m_.ce[a][s][q];
                P.bh[a][s][q] = m_.bh[a][s][q]; P.ch[a][s][q] = m_.ch[a][s][q];
            }
    }
    // psi arrays: slab axis a, depth npml, the two other axes in storage extents
    for (int c = 0; c < 3; c++)
        for (int a = 0; a < 3; a++) {
            if (a == c) continue;
            for (int s = 0; s < 2; s++) {
                int n = d.npml[a][s];
                if (n <= 0) continue;
                size_t e0 = a == 0 ? n : P.PX, e1 = a == 1 ? n : P.SY, e2 = a == 2 ? n : P.SZ;
                size_t bytes = e0 * e1 * e2 * es_;
                P.psi_h[c][a][s] = alloc(bytes);
                P.psi_e[c][a][s] = alloc(bytes);
            }
        }
    P.nmat = (int)m_.mats.size();
    P.npoles = m_.npoles;
    P.has_drude = m_.has_drude ? 1 : 0;
    P.mat = (const AemMaterial*)upload(m_.mats);
    P.ucoef = (const AemUniformCoef*)upload(m_.ucoef);
    for (int c = 0; c < 3; c++) {
        for (int q = 0; q < 6; q++) P.dbox[c][q] = m_.dbox[c][q];
        if (!m_.has_drude) continue;
        const int* b = m_.dbox[c];
        const int lo[3] = {b[4], b[2], b[0]}, hi[3] = {b[5], b[3], b[1]};
        size_t vol = 1;
        for (int a = 0; a < 3; a++) {
            if (d.pbc[a]) { P.jorg[c][a] = 0; P.jext[c][a] = m_.S[a]; }
            else { P.jorg[c][a] = lo[a] - 1; P.jext[c][a] = hi[a] >= lo[a] ? hi[a] - lo[a] + 1 : 0; }
            vol *= (size_t)P.jext[c][a];
        }
        P.jsrc[c] = alloc(vol * (size_t)m_.npoles * es_);
    }
    P.nsheet = (int)m_.splanes.size();
    for (int s = 0; s < P.nsheet; s++) {
        const SheetPlaneHost& h = m_.splanes[s];
        AemSheetPlane& S = P.sheet[s];
        S.axis = h.axis;
        S.pos = m_.pos(h.axis, h.pos);
        S.pa = h.pa; S.na = h.na; S.nb = h.nb;
        S.nmask = (const uint8_t*)upload(h.nmask);
        S.tmask = (const uint8_t*)upload(h.tmask);
        S.sa = (const float*)upload(h.sa); S.sb = (const float*)upload(h.sb);
        S.ga1 = (const float*)upload(h.ga1); S.gb1 = (const float*)upload(h.gb1);
        S.ga2 = (const float*)upload(h.ga2); S.gb2 = (const float*)upload(h.gb2);
        S.es = alloc((size_t)h.na * h.nb * es_);
    }
    P.sheet_thick = d.sheet_thickness;
    P.tfsf_on = (!d.kmax && d.pw_amp > 0) ? 1 : 0;
    P.mirror_on = (P.tfsf_on && d.is_mirror) ? 1 : 0;
    for (int a = 0; a < 3; a++) {
        P.lo[a] = d.lo[a]; P.hi[a] = d.hi[a];
        P.wall_lo[a] = d.wall_lo[a]; P.wall_hi[a] = d.wall_hi[a];
        P.coef_h[a] = d.del_t / (mu0 * dl[a]);
        P.coef_e[a] = d.del_t / (ep0 * dl[a]);
    }
    P.t_spread = d.t_spread;
    P.spread = d.spread;
    P.exp_half = std::exp(0.5f);
    P.inv_c = 1.0f / c0;
    P.pulse_type = d.pulse_type;
    for (int a = 0; a < 3; a++) {
        P.WE[0][a] = d.WE[a]; P.WH[0][a] = d.WH[a];
        P.WE[1][a] = d.WE_m[a]; P.WH[1][a] = d.WH_m[a];
        P.delay[0][a] = d.delay[a]; P.delay[1][a] = d.delay_m[a];
    }
    const float th[2] = {d.theta, d.theta_m}, ph[2] = {d.phi, d.phi_m};
    for (int m = 0; m < 2; m++) {
        P.sc[m][0] = std::sin(th[m]) * std::cos(ph[m]);
        P.sc[m][1] = std::sin(th[m]) * std::sin(ph[m]);
        P.sc[m][2] = std::cos(th[m]);
    }
    if (d.kmax) {
        for (int a = 0; a < 3; a++)
            if (d.pbc[(a + 1) % 3] && d.pbc[(a + 2) % 3] && !d.pbc[a]) P.kmax_src_axis = a;
        P.kmax_mode_TE = (d.mode_type == 0 && d.pw_amp > 0) ? 1 : 0;
        P.kmax_mode_TM = (d.mode_type == 1 && d.pw_amp > 0) ? 1 : 0;
        P.k_pl_H = d.k_pl_H;
        P.k_pl_E = d.k_pl_E;
        for (int a = 0; a < 3; a++) { P.kcnt[a] = d.kc[a]; P.knum[a] = d.knum[a]; }
        P.two_pi_f = (2.0f * pi) * d.f_adj;
    }
}

// E_or_V_1D of the standard solver, ref :8844-8857
static float eorv_std(const Deck& d, float amp, float tc, float posd) {
    const float c0 = 299792458.0f;
    float a = (d.t_spread - ((tc - 1.0f) * d.del_t) - 1.0f / c0 * posd) / d.spread;
    if (d.pulse_type == 1) return amp * std::exp(-0.5f * (a * a));
    if (d.pulse_type == 2) return amp * -1.0f * a * std::exp(0.5f) * std::exp(-0.5f * (a * a));
    return 0.0f;
}
// E_or_V_1D of the kmax solver, ref :8889-8902
static std::complex<float> eorv_kmax(const Deck& d, float amp, float tc, float posd) {
    const float c0 = 299792458.0f, pi = 3.14159265358979323846f;
    float a = (d.t_spread - ((tc - 1.0f) * d.del_t) - 1.0f / c0 * posd) / d.spread;
    float env = amp * std::exp(-0.5f * (a * a));
    float ph = 2.0f * pi * d.f_adj * ((tc - 1.0f) * d.del_t - 1.0f / c0 * posd);
    return env * std::complex<float>(std::cos(ph), std::sin(ph));
}

void Solver::setup_ports() {
    const Deck& d = m_.d;
    PortSet& S = PS_;
    std::memset(&S, 0, sizeof S);
    S.n = (int)d.ports.size();
    if (S.n > AEM_MAX_PORTS) throw DeckError("too many ports");
    S.P = d.port_array_size;
    const float dl[3] = {d.dx, d.dy, d.dz};
    // reference gridded_feed_all(num_ports,4,M1,M2) for the normalisation read
    const int M1 = m_.feed_m1, M2 = m_.feed_m2, np = S.n > 0 ? S.n : 1;
    std::vector<float> big((size_t)np * 4 * M1 * M2, 0.0f);
    for (int q = 0; q < S.n; q++) {
        const Port& p = d.ports[q];
        if (!p.gridded) continue;
        int n1 = (int)p.size[0], n2 = (int)p.size[1];
        for (int b = 1; b <= n2 + 1; b++)
            for (int a = 1; a <= n1 + 1; a++)
                for (int c = 1; c <= 4; c++)
                    big[(size_t)q + (size_t)np * ((c - 1) + 4 * ((a - 1) + (size_t)M1 * (b - 1)))] =
                        m_.feeds[q][((size_t)(b - 1) * (n1 + 1) + (a - 1)) * 4 + (c - 1)];
    }
    for (int q = 0; q < S.n; q++) {
        const Port& p = d.ports[q];
        PortDev& o = S.p[q];
        o.gridded = p.gridded;
        o.dir = p.dir;
        o.side = p.side;
        for (int a = 0; a < 3; a++) {
            o.loc[a] = (int)p.loc[a];
            o.size[a] = (int)p.size[a];
            o.sizef[a] = p.size[a];
            o.dl[a] = dl[a];
        }
        const float st = dl[p.dir];
        o.cI = (1.0f / p.L) * (d.del_t / st);
        o.cV = (1.0f / p.C) * (d.del_t / st);
        o.cS = (1.0f / std::sqrt(p.C * p.L)) * (d.del_t / st);
        o.excite = (q + 1 == d.exc_port) ? 1 : 0;
        o.V = alloc((size_t)S.P * es_);
        o.I = alloc((size_t)(S.P > 1 ? S.P - 1 : 1) * es_);
        o.vout = alloc((size_t)d.steps * es_);
        if (p.gridded) {
            o.n1 = (int)p.size[0];
            o.n2 = (int)p.size[1];
            o.feed = (const float*)upload(m_.feeds[q]);
            // ref :4948-4953, including its jj+1 read through the array's
            // column-major layout (0 past the end)
            float norm = 0.0f;
            for (int a = 1; a <= o.n1 + 1; a++)
                for (int b = 1; b <= o.n2 + 1; b++) {
                    size_t off3 = (size_t)q + (size_t)np * (2 + 4 * ((size_t)a + (size_t)M1 * (b - 1)));
                    float g3 = off3 < big.size() ? big[off3] : 0.0f;
                    float g4 = big[(size_t)q + (size_t)np * (3 + 4 * ((a - 1) + (size_t)M1 * (b - 1)))];
                    norm = norm + g3 * g3 + g4 * g4;
                }
            o.feed_norm = norm;
        }
    }
    // excitation waveforms per step, computed once on the host
    if (S.n > 0) {
        int e = d.exc_port >= 1 && d.exc_port <= S.n ? d.exc_port - 1 : 0;
        const float st = dl[d.ports[e].dir];
        if (!d.kmax) {
            std::vector<float> si(d.steps), sv(d.steps);
            for (int n = 1; n <= d.steps; n++) {
                si[n - 1] = eorv_std(d, d.ant_amp, (float)n, 0.0f * st);
                sv[n - 1] = eorv_std(d, d.ant_amp, (float)n + 0.5f, 0.5f * st);
            }
            S.srcI = upload(si);
            S.srcV = upload(sv);
        } else {
            std::vector<std::complex<float>> si(d.steps), sv(d.steps);
            for (int n = 1; n <= d.steps; n++) {
                si[n - 1] = eorv_kmax(d, d.ant_amp, (float)n, 0.0f * st);
                sv[n - 1] = eorv_kmax(d, d.ant_amp, (float)n + 0.5f, 0.5f * st);
            }
            S.srcI = upload(si);
            S.srcV = upload(sv);
        }
    }
}

void Solver::setup_farfield() {
    const Deck& d = m_.d;
    FarFieldDev& F = FF_;
    std::memset(&F, 0, sizeof F);
    F.nang = d.n_ff;
    F.len = d.len_ff + 2;
    for (int a = 0; a < 3; a++) {
        F.lo[a] = d.ff_lo[a];
        F.hi[a] = d.ff_hi[a];
        F.wall_lo[a] = d.wall_lo[a];
        F.wall_hi[a] = d.wall_hi[a];
        F.mir_off[a] = d.mir_off[a];
        F.use_mir[a] = d.use_mir[a];
        F.M_mir[a] = d.M_mir[a];
        F.J_mir[a] = d.J_mir[a];
        F.kc3[a] = d.kc[a];
    }
    F.ic = d.ic; F.jc = d.jc; F.kc = d.kc_;
    if (F.nang == 0) return;
    const float c0 = 299792458.0f, pi = 3.14159265358979323846f;
    F.r_relay = d.r_relay;
    F.c_dt = c0 * d.del_t;
    const float dl[3] = {d.dx, d.dy, d.dz};
    for (int a = 0; a < 3; a++) {
        int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
        F.fac[a] = dl[b] * dl[c] / (4.0f * pi * d.del_t * c0);
        F.has[a] = !d.pbc[a];
        // an inverted box (grid smaller than PML + TF/SF buffer) has empty
        // faces, as the reference's loops over it are empty
        const long long nb = F.hi[b] - F.lo[b] + 1, nc = F.hi[c] - F.lo[c] + 1;
        F.face_n[a] = (F.has[a] && nb > 0 && nc > 0 && F.hi[a] >= F.lo[a]) ? nb * nc : 0;
        for (int s = 0; s < 2; s++)
            if (F.has[a]) F.cur[a][s] = alloc((size_t)F.face_n[a] * 8 * es_);
    }
    F.mirror = (d.is_mirror && d.pbc[0] + d.pbc[1] + d.pbc[2] < 2 && !d.kmax) ? 1 : 0;
    std::vector<float> ang((size_t)4 * F.nang);
    for (int q = 0; q < F.nang; q++) {
        ang[4 * q + 0] = std::sin(d.ff_theta[q]);
        ang[4 * q + 1] = std::cos(d.ff_theta[q]);
        ang[4 * q + 2] = std::sin(d.ff_phi[q]);
        ang[4 * q + 3] = std::cos(d.ff_phi[q]);
    }
    F.ang = (const float*)upload(ang);
    F.UW = alloc((size_t)6 * F.nang * F.len * es_);
}

void Solver::setup_taps() {
    const Deck& d = m_.d;
    TapDev& T = TP_;
    std::memset(&T, 0, sizeof T);
    const int np = d.pbc[0] + d.pbc[1] + d.pbc[2];
    if (np == 2 || d.kmax) {
        for (int a = 0; a < 3; a++)
            if (!d.pbc[a] && d.pbc[(a + 1) % 3] && d.pbc[(a + 2) % 3]) { T.axis = a; T.plane_sum = 1; }
        if (T.plane_sum) {
            T.refl = alloc((size_t)d.steps * es_);
            T.trans = alloc((size_t)d.steps * es_);
            if (d.kmax) {
                T.refl_tm = alloc((size_t)d.steps * es_);
                T.trans_tm = alloc((size_t)d.steps * es_);
                for (int a = 0; a < 3; a++) T.knum[a] = d.knum[a];
            }
            // projection weights of the standard solver, ref :7022-7089
            const float sp = std::sin(d.pol), cp = std::cos(d.pol), sph = std::sin(d.phi), cph = std::cos(d.phi), ct = std::cos(d.theta);
            if (T.axis == 0) { T.w1 = sp; T.w2 = cp * cph; }
            if (T.axis == 1) { T.w1 = sp; T.w2 = cp * sph; }
            if (T.axis == 2) { T.w1 = (-1.0f * cp * cph - sp * ct * sph); T.w2 = (cp * sph - sp * ct * cph); }
        }
    }
    if (d.n_ff > 0 && d.pw_amp > 0) {
        T.ff_pc = 1;
        T.ic = d.ic; T.jc = d.jc; T.kc = d.kc_;
        for (int q = 0; q < 6; q++) T.pc[q] = alloc((size_t)(d.steps + 1) * es_);
    }
    if (d.video_on) {
        T.video = 1;
        T.slice_dir = d.slice_dir;
        T.slice_loc = d.slice_loc;
        T.v1 = d.vid1;
        T.v2 = d.vid2;
        for (int q = 0; q < 6; q++) T.vid[q] = alloc((size_t)T.v1 * T.v2 * d.steps * es_);
    }
}

void Solver::step(int counter) {
    launch_update_h(P_, counter, stream_);
    launch_ports_h(P_, PS_, counter, stream_);
    launch_update_e(P_, counter, stream_);
    launch_ports_e(P_, PS_, counter, stream_);
    launch_ff_currents(P_, FF_, stream_);
    launch_ff_bin(P_, FF_, counter, stream_);
    launch_taps(P_, TP_, FF_, counter, m_.d.steps, stream_);
}

void Solver::run(int n) {
    for (int q = 0; q < n && done_ < m_.d.steps; q++) {
        done_++;
        step(done_);
    }
    AEM_CUDA(cudaGetLastError());
}

}  // namespace aem
