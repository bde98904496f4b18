// aem_solver.cu -- device state and time loop of one run.
//
// The time loop order follows main_fdtd/fdtd_solver.f90:4440-8299:
//   H update (+sheets, TF/SF, CPML, PBC)  -> port H half-step
//   E update (+sheets, Drude, TF/SF, CPML, PBC) -> port E half-step
//   far-field currents and binning, plane sums, phase-centre, video.
#include "aem_solver.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>

namespace aem {

#define AEM_CUDA(x)                                                                                     \
    do {                                                                                                \
        cudaError_t e_ = (x);                                                                           \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + \
                                                        " at " #x);                                     \
    } while (0)

static bool getenv_flag(const char* name) {
    const char* v = std::getenv(name);
    return v && *v && std::strcmp(v, "0") != 0;
}

static std::string dir_of(const std::string& p) {
    size_t s = p.find_last_of('/');
    return s == std::string::npos ? std::string() : p.substr(0, s);
}

void* Solver::alloc(size_t bytes) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    // fault injection: AEM_FAIL_ALLOC_AT=n fails the n-th allocation of this
    // handle as if the device were out of memory (host-side; tests the
    // error path and the release of what was allocated before)
    if (const char* v = std::getenv("AEM_FAIL_ALLOC_AT"))
        if (std::atol(v) == (long)bufs_.size() + 1)
            throw std::runtime_error("CUDA error: out of memory (injected by AEM_FAIL_ALLOC_AT) allocating " +
                                     std::to_string(bytes) + " bytes");
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();  // do not leave the failure pending for later calls
        throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e) + " allocating " +
                                 std::to_string(bytes) + " bytes");
    }
    AEM_CUDA(cudaMemsetAsync(p, 0, bytes, stream_));
    bufs_.push_back(p);
    buf_bytes_.push_back(bytes);
    dev_bytes_ += bytes;
    return p;
}

template <typename V, typename A>
void* Solver::upload(const std::vector<V, A>& v) {
    void* p = alloc(v.size() * sizeof(V));
    if (!v.empty()) AEM_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice, stream_));
    h2d_bytes_ += v.size() * sizeof(V);
    return p;
}

Solver::Solver(const std::string& inputs_path, bool kmax, const std::string& outdir) : outdir_(outdir) {
    m_.d = parse_deck_file(inputs_path, kmax);
    derive(m_.d);
    build_model(m_, dir_of(inputs_path));
    init();
}

Solver::Solver(const std::string& deck_text, const std::string& ext_text, const float* bulk, size_t bulk_n, bool kmax,
               const std::string& outdir, const std::string& workdir)
    : outdir_(outdir) {
    m_.d = parse_deck(deck_text, kmax);
    apply_extensions(m_.d, ext_text);
    derive(m_.d);
    build_model(m_, workdir, bulk, bulk_n);
    init();
}

void Solver::init() {
    try {
        AEM_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        es_ = m_.d.kmax ? 8 : 4;
        setup_params();
        setup_ports();
        setup_farfield();
        setup_taps();
        setup_full();
        setup_fused();
        AEM_CUDA(cudaStreamSynchronize(stream_));
        nstate_ = bufs_.size();
        // scratch, not run state, allocated after the state buffers so that
        // checkpoints neither hold nor depend on it: the watchdog flag and
        // the far-field window sums of one batch
        if (m_.d.ext_watchdog > 0) wd_flag_ = (int*)alloc(sizeof(int));
        if (ff_part_bytes_) FF_.part = (float*)alloc(ff_part_bytes_);
    } catch (...) {
        release();  // a throwing constructor runs no destructor
        throw;
    }
}

// the fused H+E kernel needs second field and H-psi buffers (ping-pong)
void Solver::setup_fused() {
    int gridded = 0;
    for (int q = 0; q < PS_.n; q++) gridded += PS_.p[q].gridded;
    // a port whose cells or H loop reach a CPML slab sees the fields between
    // the bulk pass and the CPML pass, as in the reference (ports_h before
    // cpml_h, ports_e before cpml_e, ref :4797-5375 / :6120-6670)
    const Deck& dk = m_.d;
    const int N[3] = {dk.X, dk.Y, dk.Z};
    split_ = false;
    for (const Port& pt : dk.ports) {
        if (pt.gridded) { split_ = true; continue; }  // feed planes: keep the reference order always
        for (int a = 0; a < 3; a++) {
            if (dk.pbc[a]) continue;
            const int lo = (int)pt.loc[a] - 1, hi = (int)pt.loc[a] + (int)pt.size[a];
            if (lo <= dk.npml[a][0] || hi >= N[a] + 1 - dk.npml[a][1]) split_ = true;
        }
    }
    fused_ = yee_fused_ok(P_, gridded) && !split_ && !getenv_flag("AEM_TWO_KERNEL");
    if (!fused_) return;
    P_.err = (int*)alloc(sizeof(int));
    for (int c = 0; c < 3; c++) {
        P_.E2[c] = alloc((size_t)m_.cells * es_);
        P_.H2[c] = alloc((size_t)m_.cells * es_);
    }
    for (int c = 0; c < 3; c++)
        for (int a = 0; a < 3; a++)
            for (int s = 0; s < 2; s++) {
                if (!P_.psi_h[c][a][s]) continue;
                int n = dk.npml[a][s];
                size_t e0 = a == 0 ? n : P_.PX, e1 = a == 1 ? n : P_.SY, e2 = a == 2 ? n : P_.SZ;
                P_.psi_h2[c][a][s] = alloc(e0 * e1 * e2 * es_);
            }
}

void Solver::release() {
    if (stream_) cudaStreamSynchronize(stream_);
    // steps already run still reach the export files (nothing is written if
    // the device is in an error state)
    try {
        full_flush();
    } catch (...) {
    }
    for (int q = 0; q < 6; q++) {
        if (full_.f[q]) std::fclose(full_.f[q]);
        full_.f[q] = nullptr;
    }
    for (int b = 0; b < 2; b++) {
        if (full_.host[b]) cudaFreeHost(full_.host[b]);
        if (full_.made[b]) cudaEventDestroy(full_.made[b]);
        if (full_.copied[b]) cudaEventDestroy(full_.copied[b]);
        full_.host[b] = nullptr;
        full_.made[b] = full_.copied[b] = nullptr;
        full_.pending[b] = 0;
    }
    if (full_.copy) cudaStreamDestroy(full_.copy);
    full_.copy = nullptr;
    release_graph();
    for (void* p : bufs_) cudaFree(p);
    bufs_.clear();
    buf_bytes_.clear();
    for (cudaEvent_t e : prof_pool_) cudaEventDestroy(e);
    prof_pool_.clear();
    if (stream_) cudaStreamDestroy(stream_);
    stream_ = nullptr;
}

Solver::~Solver() { release(); }

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
    P.zch_h = P.zch_e = 16;  // two-kernel launch shape until autotune picks one
    P.ty_h = P.ty_e = 8;
    for (int c = 0; c < 3; c++) {
        P.E[c] = alloc((size_t)m_.cells * es_);
        P.H[c] = alloc((size_t)m_.cells * es_);
    }
    if (m_.raster_device) {
        uint8_t* ids = (uint8_t*)alloc((size_t)m_.cells);  // zeroed on stream_
        rasterise_device(m_, ids, stream_, h2d_bytes_);
        P.cell = ids;
        m_.raster_bulk = nullptr;  // the caller's buffer is not kept
        std::vector<float>().swap(m_.raster_file);
    } else {
        P.cell = (const uint8_t*)upload(m_.cell_id);
    }
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
    // TF/SF faces (H: lo-1 and hi, E: lo and hi, over lo-1..hi on the other
    // axes) clear of every CPML slab: the corrections can follow the update
    // in their own kernels, since no CPML term reaches those positions
    P.tfsf_sep = 0;
    if (P.tfsf_on) {
        bool sep = true;
        for (int a = 0; a < 3; a++) {
            if (d.pbc[a]) { sep &= d.npml[a][0] == 0 && d.npml[a][1] == 0; continue; }
            sep &= d.lo[a] - 1 >= d.npml[a][0] && d.hi[a] <= N[a] - d.npml[a][1] && d.lo[a] - 1 >= 1 && d.hi[a] >= d.lo[a];
        }
        P.tfsf_sep = sep && !getenv_flag("AEM_TFSF_INLINE") ? 1 : 0;  // the switch: for comparisons
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
        // a face whose tangential range is inverted (grid smaller than PML +
        // buffer along that axis) is empty, as the reference's loops over it
        // are; an inverted range along the normal still has its two planes
        // (the reference visits ff_low and ff_high whatever their order)
        const long long nb = F.hi[b] - F.lo[b] + 1, nc = F.hi[c] - F.lo[c] + 1;
        F.face_n[a] = (F.has[a] && nb > 0 && nc > 0) ? nb * nc : 0;
        F.tiles_u[a] = F.face_n[a] ? (int)((nb + FF_TILE - 1) / FF_TILE) : 0;
        F.tiles_v[a] = F.face_n[a] ? (int)((nc + FF_TILE - 1) / FF_TILE) : 0;
    }
    F.mirror = (d.is_mirror && d.pbc[0] + d.pbc[1] + d.pbc[2] < 2 && !d.kmax) ? 1 : 0;
    F.nvang = F.nang * (1 + F.mirror);
    std::vector<float> ang((size_t)4 * F.nang);
    for (int q = 0; q < F.nang; q++) {
        ang[4 * q + 0] = std::sin(d.ff_theta[q]);
        ang[4 * q + 1] = std::cos(d.ff_theta[q]);
        ang[4 * q + 2] = std::sin(d.ff_phi[q]);
        ang[4 * q + 3] = std::cos(d.ff_phi[q]);
    }
    F.ang = (const float*)upload(ang);
    // accumulators: FP64 (deterministic ordered sums); a constant-k run
    // keeps a real and an imaginary plane
    F.UW = alloc((size_t)6 * F.nang * F.len * sizeof(double) * (d.kmax ? 2 : 1));
    F.err = (int*)alloc(sizeof(int));

    // retarded-time offset of face cell (u, v) for virtual angle va (image
    // pass second): tf = (r_relay - sum_e (pos_e - centre_e) del_e dir_e) / (c dt)
    // with pos the cell's reference index (mirrored in the image pass,
    // ref :7958-8230), written as K0 + Ku u + Kv v
    std::vector<float> kf((size_t)F.nvang * 3 * 2 * 3, 0.0f);
    const int ctr[3] = {F.ic, F.jc, F.kc};
    for (int va = 0; va < F.nvang; va++) {
        const int q = va % F.nang, pass = va / F.nang;
        const double dir[3] = {(double)ang[4 * q] * ang[4 * q + 3], (double)ang[4 * q] * ang[4 * q + 2], (double)ang[4 * q + 1]};
        for (int a = 0; a < 3; a++) {
            const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
            for (int s = 0; s < 2; s++) {
                // pos_e = sg_e * idx_e + of_e
                double sg[3], of[3];
                for (int e = 0; e < 3; e++) {
                    const bool m = pass && F.use_mir[e] != 0.0f;
                    sg[e] = m ? -1.0 : 1.0;
                    of[e] = m ? (double)F.mir_off[e] : 0.0;
                }
                int idx0[3];
                idx0[a] = s ? F.hi[a] : F.lo[a];
                idx0[b] = F.lo[b];
                idx0[c] = F.lo[c];
                double proj0 = 0;
                for (int e = 0; e < 3; e++) proj0 += (sg[e] * idx0[e] + of[e] - ctr[e]) * (double)dl[e] * dir[e];
                float* k = &kf[(((size_t)va * 3 + a) * 2 + s) * 3];
                k[0] = (float)(((double)F.r_relay - proj0) / (double)F.c_dt);
                k[1] = (float)(-sg[b] * (double)dl[b] * dir[b] / (double)F.c_dt);
                k[2] = (float)(-sg[c] * (double)dl[c] * dir[c] / (double)F.c_dt);
            }
        }
    }
    // angles of one direction (the poles theta = 0, 180 at every phi) have the
    // same delays on every face and pass, so the same bins of the Cartesian
    // components: the batched path bins the first such angle and the others
    // copy its bins when the output is written
    ff_canon_.resize(F.nang);
    {
        std::map<std::string, int> first;
        const size_t per = (size_t)3 * 2 * 3;
        for (int q = 0; q < F.nang; q++) {
            std::string key;
            for (int pass = 0; pass <= F.mirror; pass++)
                key.append(reinterpret_cast<const char*>(&kf[(size_t)(q + pass * F.nang) * per]), per * sizeof(float));
            ff_canon_[q] = first.emplace(key, q).first->second;
        }
    }
    // batches of FF_TB steps, binned deterministically over 32x32 face tiles
    // (aem_ffbin.cu); a constant-k run bins its real and imaginary planes
    F.tb = FF_TB;
    {
        F.kf = (const float*)upload(kf);
        F.tile0[0] = 0;
        for (int f = 0; f < 6; f++) F.tile0[f + 1] = F.tile0[f] + (long long)F.tiles_u[f >> 1] * F.tiles_v[f >> 1];
        F.ntiles = (int)F.tile0[6];
        F.maxt = 0;
        for (int f = 0; f < 6; f++) F.maxt = std::max(F.maxt, (int)(F.tile0[f + 1] - F.tile0[f]));
        // binned virtual angles: those of canonical directions; j of each
        std::vector<int> vlist, jof(F.nvang, -1);
        for (int va = 0; va < F.nvang; va++)
            if (ff_canon_[va % F.nang] == va % F.nang) {
                jof[va] = (int)vlist.size();
                vlist.push_back(va);
            }
        F.nvc = (int)vlist.size();
        F.vlist = (const int*)upload(vlist);
        if (F.ntiles > 0 && F.nvc > 0) {
            // window bases and spans, from the binning kernel's own expressions
            int* kb_d = (int*)alloc((size_t)F.ntiles * F.nvc * sizeof(int));
            int* span_d = (int*)alloc(sizeof(int));
            launch_ff_base(F, kb_d, span_d, stream_);
            std::vector<int> kb((size_t)F.ntiles * F.nvc);
            int span = 0;
            AEM_CUDA(cudaMemcpyAsync(kb.data(), kb_d, kb.size() * sizeof(int), cudaMemcpyDeviceToHost, stream_));
            AEM_CUDA(cudaMemcpyAsync(&span, span_d, sizeof(int), cudaMemcpyDeviceToHost, stream_));
            AEM_CUDA(cudaStreamSynchronize(stream_));
            AEM_CUDA(cudaGetLastError());
            F.kb = kb_d;
            F.hs = span + FF_TB + 1;  // offsets base .. base+span, plus the 32 lanes and the final step's carry
            // angles per CTA: 8 warps x AW, two CTAs per SM
            const size_t stage = (size_t)2 * FF_TILE * (4 * 33 + 1) * sizeof(float);
            const size_t per = (size_t)2 * F.hs * 2 * sizeof(float);
            F.group = 8;
            if (stage + 32 * per <= 96 * 1024) F.group = 32;
            else if (stage + 16 * per <= 96 * 1024) F.group = 16;
            if (stage + F.group * per > 200 * 1024)
                throw std::runtime_error("far field: a tile's delay span (" + std::to_string(span) +
                                         " steps) is too wide for the binning windows");
            F.ngrp = (F.nvc + F.group - 1) / F.group;
            // per (j, face): tiles sorted by (kb, tile), for the ordered reduction
            std::vector<int> srt((size_t)F.nvc * 6 * F.maxt, 0), srtkb((size_t)F.nvc * 6 * F.maxt, INT_MAX);
            std::vector<int> kbmin((size_t)F.nvc, INT_MAX), kbmax((size_t)F.nvc, INT_MIN);
            par_for(F.nvc, [&](int j) {  // each angle writes its own lists
                std::vector<int> idx;
                for (int f = 0; f < 6; f++) {
                    const int t0 = (int)F.tile0[f], nt = (int)(F.tile0[f + 1] - F.tile0[f]);
                    idx.resize(nt);
                    for (int q = 0; q < nt; q++) idx[q] = t0 + q;
                    std::sort(idx.begin(), idx.end(), [&](int x, int y) {
                        const int kx = kb[(size_t)x * F.nvc + j], ky = kb[(size_t)y * F.nvc + j];
                        return kx != ky ? kx < ky : x < y;
                    });
                    const size_t o = ((size_t)j * 6 + f) * F.maxt;
                    for (int q = 0; q < nt; q++) {
                        srt[o + q] = idx[q];
                        srtkb[o + q] = kb[(size_t)idx[q] * F.nvc + j];
                    }
                    if (nt) {
                        kbmin[j] = std::min(kbmin[j], srtkb[o]);
                        kbmax[j] = std::max(kbmax[j], srtkb[o + nt - 1]);
                    }
                }
            });
            F.srt = (const int*)upload(srt);
            F.srtkb = (const int*)upload(srtkb);
            // reduction CTAs: the canonical angles, with the j of each pass
            std::vector<int> clist, crange;
            for (int q = 0; q < F.nang; q++) {
                if (ff_canon_[q] != q) continue;
                const int j0 = jof[q], j1 = F.mirror ? jof[q + F.nang] : -1;
                int lo = INT_MAX, hi = INT_MIN;
                for (int j : {j0, j1})
                    if (j >= 0) { lo = std::min(lo, kbmin[j]); hi = std::max(hi, kbmax[j] + F.hs); }
                if (lo > hi) lo = hi = 0;
                clist.insert(clist.end(), {q, j0, j1, 0});
                crange.insert(crange.end(), {lo, hi});
            }
            F.nangc = (int)clist.size() / 4;
            F.clist = (const int*)upload(clist);
            F.crange = (const int*)upload(crange);
            F.dtile = (float*)alloc((size_t)F.ntiles * FF_SLOTS * 4 * 1024 * sizeof(float) * (d.kmax ? 2 : 1));
            ff_part_bytes_ = (size_t)F.ntiles * F.nvc * 4 * F.hs * sizeof(float);
            ff_tiles_prepare();
        }
    }
    for (int a = 0; a < 3; a++)
        for (int s = 0; s < 2; s++)
            if (F.has[a]) F.cur[a][s] = alloc((size_t)F.face_n[a] * 4 * es_);
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
    if (!d.ext_probes.empty()) {
        const int n[3] = {d.nx, d.ny, d.nz};
        T.nprobe = (int)d.ext_probes.size();
        for (int q = 0; q < T.nprobe; q++)
            for (int a = 0; a < 3; a++) {
                const int v = d.ext_probes[q][a];
                if (v < 1 || v > n[a])
                    throw DeckError("extension probe " + std::to_string(q + 1) + ": cell index outside 1..n on axis " +
                                    std::to_string(a));
                T.prb_idx[q][a] = v;
            }
        T.prb = alloc((size_t)3 * T.nprobe * d.steps * es_);
    }
    dft_series_.clear();
    if (!d.ext_dft_freqs.empty()) {
        // series in the order of the probe kinds: plane sums, then port voltages
        auto add = [&](int kind, int index, const void* p) {
            T.ser[dft_series_.size()] = p;
            dft_series_.push_back({kind, index});
        };
        if (T.plane_sum) {
            add(1, 0, T.refl);
            add(2, 0, T.trans);
            if (d.kmax) { add(3, 0, T.refl_tm); add(4, 0, T.trans_tm); }
        }
        for (int q = 0; q < PS_.n; q++) add(5, q, PS_.p[q].vout);
        if (dft_series_.empty())
            throw DeckError("extension dft_freqs: the deck records no per-step series (unit-cell plane sums or ports)");
        T.nser = (int)dft_series_.size();
        T.ndft = (int)d.ext_dft_freqs.size();
        T.dft_dt = (double)d.del_t;
        T.dft_f = (const double*)upload(d.ext_dft_freqs);
        T.dft_acc = (double*)alloc((size_t)T.nser * T.ndft * 2 * sizeof(double));
        T.dft_cmp = (double*)alloc((size_t)T.nser * T.ndft * 2 * sizeof(double));
    }
}

// spectrum of one per-step series over the steps run so far
int Solver::read_spectrum(int kind, int index, int n, double* freqs, double* re, double* im) {
    int sr = -1;
    for (size_t q = 0; q < dft_series_.size(); q++)
        if (dft_series_[q].first == kind && dft_series_[q].second == index) sr = (int)q;
    if (!TP_.ndft) throw std::invalid_argument("no on-the-fly spectra: the run has no dft_freqs extension");
    if (sr < 0) throw std::invalid_argument("no spectrum of that series (kind 1..4 plane sums, 5 port voltage)");
    const int nf = std::min(n, TP_.ndft);
    std::vector<double> buf((size_t)TP_.ndft * 2);
    AEM_CUDA(cudaMemcpyAsync(buf.data(), TP_.dft_acc + (size_t)sr * TP_.ndft * 2, buf.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, stream_));
    AEM_CUDA(cudaStreamSynchronize(stream_));
    d2h_bytes_ += buf.size() * sizeof(double);
    for (int f = 0; f < nf; f++) {
        if (freqs) freqs[f] = m_.d.ext_dft_freqs[f];
        re[f] = buf[2 * f];
        if (im) im[f] = buf[2 * f + 1];
    }
    return nf;
}

// Full-field export files, opened at setup like the reference's units
// 17-22 (ref :3971 allocation, :6995-7000 writes); one Fortran unformatted
// record (4-byte length, FP32 values (re, im pairs for kmax), 4-byte
// length) per component per step.
void Solver::setup_full() {
    const Deck& d = m_.d;
    if (d.export_all != "yes") return;
    const int N[3] = {d.X, d.Y, d.Z};
    size_t cells = 1;
    for (int a = 0; a < 3; a++) {
        full_.n[a] = N[a] - 1 - d.pbc[a];
        cells *= (size_t)full_.n[a];
    }
    if (cells * es_ > 0x7fffffffu)
        throw std::invalid_argument("full-field export: one component of one step exceeds the 2 GiB record length");
    full_.bytes = 6 * cells * es_;
    AEM_CUDA(cudaStreamCreateWithFlags(&full_.copy, cudaStreamNonBlocking));
    for (int b = 0; b < 2; b++) {
        full_.dev[b] = alloc(full_.bytes);
        AEM_CUDA(cudaMallocHost(&full_.host[b], full_.bytes));
        AEM_CUDA(cudaEventCreateWithFlags(&full_.made[b], cudaEventDisableTiming));
        AEM_CUDA(cudaEventCreateWithFlags(&full_.copied[b], cudaEventDisableTiming));
    }
    static const char* nm[6] = {"Ex", "Ey", "Ez", "Hx", "Hy", "Hz"};
    const std::string base = d.filename.substr(0, d.filename.size() >= 4 ? d.filename.size() - 4 : 0);
    for (int q = 0; q < 6; q++) {
        const std::string fn = (outdir_.empty() ? "" : outdir_ + "/") + base + "_full_" + nm[q] + ".bin";
        full_.f[q] = std::fopen(fn.c_str(), "wb");
        if (!full_.f[q]) throw std::runtime_error("full-field export: cannot open " + fn);
    }
}

// average step `counter` into staging buffer counter % 2 and start its copy
// to the host; the buffer's previous step (counter - 2) is written first
void Solver::full_tap(int counter) {
    const int b = counter & 1;
    if (full_.pending[b]) full_drain(b);
    phase(AEM_PHASE_TAPS, [&] { return launch_full(P_, full_.dev[b], full_.n, stream_); });
    AEM_CUDA(cudaEventRecord(full_.made[b], stream_));
    AEM_CUDA(cudaStreamWaitEvent(full_.copy, full_.made[b], 0));
    AEM_CUDA(cudaMemcpyAsync(full_.host[b], full_.dev[b], full_.bytes, cudaMemcpyDeviceToHost, full_.copy));
    AEM_CUDA(cudaEventRecord(full_.copied[b], full_.copy));
    full_.pending[b] = counter;
    d2h_bytes_ += full_.bytes;
}

// wait for buffer b's copy and append its six records to the files
void Solver::full_drain(int b) {
    AEM_CUDA(cudaEventSynchronize(full_.copied[b]));
    const size_t per = full_.bytes / 6;
    const int32_t L = (int32_t)per;
    for (int q = 0; q < 6; q++) {
        std::FILE* f = full_.f[q];
        if (std::fwrite(&L, 4, 1, f) != 1 || std::fwrite((const char*)full_.host[b] + q * per, 1, per, f) != per ||
            std::fwrite(&L, 4, 1, f) != 1)
            throw std::runtime_error("full-field export: write failed");
    }
    full_.pending[b] = 0;
}

// write every step still held in a copy buffer, oldest first
void Solver::full_flush() {
    if (!full_.f[0]) return;
    int first = 0;
    if (full_.pending[1] && (!full_.pending[0] || full_.pending[1] < full_.pending[0])) first = 1;
    for (int b : {first, 1 - first})
        if (full_.pending[b]) full_drain(b);
    for (std::FILE* f : full_.f) std::fflush(f);
}

// run one launcher; with profiling on, bracket it with events on the stream
template <typename Fn>
void Solver::phase(int ph, Fn&& fn) {
    if (!prof_on_) {
        launches_ += fn();
        return;
    }
    cudaEvent_t e0 = prof_event(), e1 = prof_event();
    AEM_CUDA(cudaEventRecord(e0, stream_));
    const int n = fn();
    AEM_CUDA(cudaEventRecord(e1, stream_));
    launches_ += n;
    if (n) prof_marks_.push_back({ph, n, e0, e1});
}

cudaEvent_t Solver::prof_event() {
    if (prof_used_ == prof_pool_.size()) {
        cudaEvent_t e;
        AEM_CUDA(cudaEventCreate(&e));
        prof_pool_.push_back(e);
    }
    return prof_pool_[prof_used_++];
}

void Solver::set_profiling(bool on) {
    AEM_CUDA(cudaStreamSynchronize(stream_));
    prof_on_ = on;
    prof_used_ = 0;
    prof_marks_.clear();
}

void Solver::read_profile(double ms[AEM_NPHASE], long long launches[AEM_NPHASE]) {
    AEM_CUDA(cudaStreamSynchronize(stream_));
    for (int p = 0; p < AEM_NPHASE; p++) { ms[p] = 0; launches[p] = 0; }
    for (const ProfMark& m : prof_marks_) {
        float t = 0;
        AEM_CUDA(cudaEventElapsedTime(&t, m.e0, m.e1));
        ms[m.phase] += t;
        launches[m.phase] += m.n;
    }
}

void Solver::read_probe(int kind, int index, int first, int n, double* re, double* im) {
    const void* src = nullptr;
    if (kind == 5) {
        if (index < 0 || index >= PS_.n) throw std::invalid_argument("no such port");
        src = PS_.p[index].vout;
    } else if (kind >= 1 && kind <= 4) {
        if (!TP_.plane_sum) throw std::invalid_argument("the deck has no reflection/transmission planes");
        if (kind >= 3 && !m_.d.kmax) throw std::invalid_argument("TM plane sums (kinds 3, 4) exist in kmax runs only");
        src = kind == 1 ? TP_.refl : kind == 2 ? TP_.trans : kind == 3 ? TP_.refl_tm : TP_.trans_tm;
    } else if (kind == 6) {
        if (index < 0 || index >= 3 * TP_.nprobe) throw std::invalid_argument("no such point probe component (index 3 p + c)");
        src = (const char*)TP_.prb + (size_t)index * m_.d.steps * es_;
    } else {
        throw std::invalid_argument("probe kind must be 1..6");
    }
    if (first < 1 || n < 0 || first - 1 + n > done_) throw std::invalid_argument("steps outside those run so far");
    std::vector<char> buf((size_t)n * es_);
    AEM_CUDA(cudaMemcpyAsync(buf.data(), (const char*)src + (size_t)(first - 1) * es_, buf.size(), cudaMemcpyDeviceToHost, stream_));
    AEM_CUDA(cudaStreamSynchronize(stream_));
    d2h_bytes_ += buf.size();
    for (int q = 0; q < n; q++) {
        if (es_ == 4) {
            re[q] = ((const float*)buf.data())[q];
            if (im) im[q] = 0;
        } else {
            re[q] = ((const float*)buf.data())[2 * q];
            if (im) im[q] = ((const float*)buf.data())[2 * q + 1];
        }
    }
}

void Solver::step(int counter) {
    if (fused_) {
        // H and E in one pass into the second buffers, then swap; the basic
        // ports read H_new and overwrite E_new exactly as between and after
        // the reference's two half-steps
        phase(AEM_PHASE_YEE, [&] { return launch_yee(P_, stream_); });
        for (int c = 0; c < 3; c++) {
            std::swap(P_.E[c], P_.E2[c]);
            std::swap(P_.H[c], P_.H2[c]);
            for (int a = 0; a < 3; a++)
                for (int s = 0; s < 2; s++) std::swap(P_.psi_h[c][a][s], P_.psi_h2[c][a][s]);
        }
        phase(AEM_PHASE_PORTS, [&] { return launch_ports_h(P_, PS_, counter, stream_); });
        phase(AEM_PHASE_PORTS, [&] { return launch_ports_e(P_, PS_, counter, stream_); });
    } else if (split_) {
        AemParams& P1 = split_params_[0];
        AemParams& P2 = split_params_[1];
        P1 = P_; P1.cpml_split = 1;
        P2 = P_; P2.cpml_split = 2;
        phase(AEM_PHASE_UPDATE_H, [&] { return launch_update_h(P1, counter, stream_); });
        phase(AEM_PHASE_PORTS, [&] { return launch_ports_h(P_, PS_, counter, stream_); });
        phase(AEM_PHASE_UPDATE_H, [&] { return launch_update_h(P2, counter, stream_); });
        phase(AEM_PHASE_UPDATE_E, [&] { return launch_update_e(P1, counter, stream_); });
        phase(AEM_PHASE_PORTS, [&] { return launch_ports_e(P_, PS_, counter, stream_); });
        phase(AEM_PHASE_UPDATE_E, [&] { return launch_update_e(P2, counter, stream_); });
    } else {
        phase(AEM_PHASE_UPDATE_H, [&] { return launch_update_h(P_, counter, stream_); });
        phase(AEM_PHASE_PORTS, [&] { return launch_ports_h(P_, PS_, counter, stream_); });
        phase(AEM_PHASE_UPDATE_E, [&] { return launch_update_e(P_, counter, stream_); });
        phase(AEM_PHASE_PORTS, [&] { return launch_ports_e(P_, PS_, counter, stream_); });
    }
    {
        // differences go to slot counter - ff_n0_ + 1; a full batch is binned at once
        phase(AEM_PHASE_FF_CURRENTS, [&] { return launch_ff_currents(P_, FF_, counter - ff_n0_ + 1, stream_); });
        if (counter == m_.d.steps && !P_.dstep) flush_farfield_last(counter);
        else if (counter - ff_n0_ + 1 == FF_.tb) flush_farfield(counter);
    }
    phase(AEM_PHASE_TAPS, [&] { return launch_taps(P_, TP_, FF_, counter, m_.d.steps, stream_); });
    if (full_.f[0]) full_tap(counter);
}

// bin the steps ff_n0_..last held in the difference buffer; the last one
// moves to slot 0, where the next batch takes its carried-over part
void Solver::flush_farfield(int last) {
    if (last < ff_n0_) return;  // nothing buffered (and the tail, if done, stays done)
    const int n0 = ff_n0_, nt = last - ff_n0_ + 1;
    bin_farfield(n0, nt, nt, false);
    ff_n0_ = last + 1;
}

// the binning launches of one batch: the real plane, and for a constant-k
// run the imaginary plane (its differences and accumulators follow the
// real ones)
void Solver::bin_farfield(int n0, int nt, int carry, bool tail) {
    phase(AEM_PHASE_FF_BIN, [&] { return launch_ff_bin_tiles(P_, FF_, n0, nt, carry, stream_, tail); });
    if (m_.d.kmax) {
        FarFieldDev Fi = FF_;
        Fi.dtile = FF_.dtile ? FF_.dtile + (size_t)FF_.ntiles * FF_SLOTS * 4 * 1024 : nullptr;
        Fi.UW = (double*)FF_.UW + (size_t)6 * FF_.nang * FF_.len;
        phase(AEM_PHASE_FF_BIN, [&] { return launch_ff_bin_tiles(P_, Fi, n0, nt, carry, stream_, tail); });
    }
}

// the deck's last step, run eagerly: its batch and the carried-over part of
// that step in one launch (a separate one-lane launch costs as much as a
// full batch); ff_n0_ then points past the tail, as flush_farfield_tail
// leaves it
void Solver::flush_farfield_last(int last) {
    const int n0 = ff_n0_, nt = last - ff_n0_ + 1;
    bin_farfield(n0, nt, -1, true);
    ff_n0_ = m_.d.steps + 2;
}

// after the deck's last step: the carried-over part of that step, binned as
// a one-step batch whose own differences are zero; ff_n0_ then points past
// it, so this runs once (a checkpoint carries ff_n0_)
void Solver::flush_farfield_tail() {
    const int steps = m_.d.steps;
    if (done_ == steps && ff_n0_ == steps + 1) {
        bin_farfield(steps + 1, 1, -1, false);
        ff_n0_ = steps + 2;
    }
}

// every K steps (extension watchdog K): scan the current E and H for a
// non-finite value; the run stops with Diverged at the first step found so
void Solver::watchdog_check() {
    FieldPtrs F;
    for (int c = 0; c < 3; c++) { F.p[c] = P_.E[c]; F.p[3 + c] = P_.H[c]; }
    launches_ += launch_nonfinite(F, (long long)m_.cells * es_ / 16, wd_flag_, stream_);
    int bad = 0;
    AEM_CUDA(cudaMemcpyAsync(&bad, wd_flag_, sizeof bad, cudaMemcpyDeviceToHost, stream_));
    AEM_CUDA(cudaStreamSynchronize(stream_));
    d2h_bytes_ += sizeof bad;
    if (bad) throw Diverged("the fields diverged: a non-finite value at step " + std::to_string(done_));
}

int Solver::autotune_pending(int budget) {
    if (tuned_ || m_.d.ext_autotune <= 0 || budget <= 0) return 0;
    const int d0 = done_;
    autotune(m_.d.ext_autotune, nullptr, budget);
    return done_ - d0;
}

void Solver::autotune(int per, int out[4], int budget) {
    struct Shape {
        int zch, ty;
    };
    // z planes per CTA, rows per CTA (32 columns each)
    static const Shape cand[] = {{16, 8}, {8, 8}, {32, 8}, {4, 8}, {64, 8}, {16, 4}, {8, 4}, {32, 4}};
    const int ncand = (int)(sizeof cand / sizeof cand[0]);
    tuned_ = true;  // first: the tuning steps below go through run()
    if (!fused_ && per > 0) {
        const bool prof = prof_on_;
        double best_h = 1e300, best_e = 1e300;
        Shape bh = {P_.zch_h, P_.ty_h}, be = {P_.zch_e, P_.ty_e};
        const int d0 = done_;
        for (int c = 0; c < ncand && done_ + per <= m_.d.steps && done_ - d0 + per <= budget; c++) {
            P_.zch_h = P_.zch_e = cand[c].zch;
            P_.ty_h = P_.ty_e = cand[c].ty;
            set_profiling(true);
            run(per);
            double ms[AEM_NPHASE];
            long long nl[AEM_NPHASE];
            read_profile(ms, nl);
            // per launch (the split CPML order launches each kernel twice a step)
            const double th = nl[AEM_PHASE_UPDATE_H] ? ms[AEM_PHASE_UPDATE_H] / nl[AEM_PHASE_UPDATE_H] : 1e300;
            const double te = nl[AEM_PHASE_UPDATE_E] ? ms[AEM_PHASE_UPDATE_E] / nl[AEM_PHASE_UPDATE_E] : 1e300;
            if (th < best_h) { best_h = th; bh = cand[c]; }
            if (te < best_e) { best_e = te; be = cand[c]; }
        }
        P_.zch_h = bh.zch; P_.ty_h = bh.ty;
        P_.zch_e = be.zch; P_.ty_e = be.ty;
        set_profiling(prof);
        release_graph();  // a captured graph holds the old shape
    }
    if (out) {
        out[0] = P_.zch_h; out[1] = P_.ty_h;
        out[2] = P_.zch_e; out[3] = P_.ty_e;
    }
}

void Solver::run(int n) {
    n -= autotune_pending(n);  // extension autotune: the tuning steps count towards n
    const int K = m_.d.ext_watchdog;
    for (int q = 0; q < n && done_ < m_.d.steps; q++) {
        done_++;
        step(done_);
        if (K > 0 && done_ % K == 0) watchdog_check();
    }
    // the last step bins whatever the batch buffer still holds; earlier
    // partial batches wait for more steps (or for flush())
    if (done_ == m_.d.steps) {
        flush_farfield(done_);
        flush_farfield_tail();
        full_flush();
    }
    AEM_CUDA(cudaGetLastError());
}

void Solver::release_graph() {
    if (graph_) cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
    graph_g_ = 0;
}

bool Solver::graph_ready(int g) const {
    if (g < 1 || done_ == 0 || done_ + g > m_.d.steps) return false;  // the first step runs eagerly
    if (full_.f[0]) return false;                                       // the host writes every step's export
    if (fused_ && (g & 1)) return false;                                // an even number of buffer swaps
    if (FF_.tb > 1 && (g % FF_.tb != 0 || ff_n0_ != done_ + 1)) return false;  // whole far-field batches
    return true;
}

// Record g steps (each followed by the counter advance) on the solver's
// stream without running them; the host-side state the recording moved on
// (far-field batch start, launch count) is put back, replays move it.
void Solver::capture_graph(int g) {
    release_graph();
    if (!dstep_) dstep_ = (int*)alloc(sizeof(int));
    const int n0 = ff_n0_;
    const long long l0 = launches_;
    const bool prof = prof_on_;
    prof_on_ = false;
    P_.dstep = dstep_;
    cudaGraph_t graph = nullptr;
    AEM_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    try {
        for (int q = 1; q <= g; q++) {
            step(done_ + q);
            launches_ += launch_step_advance(dstep_, stream_);
        }
    } catch (...) {
        cudaStreamEndCapture(stream_, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        P_.dstep = nullptr;
        ff_n0_ = n0;
        launches_ = l0;
        prof_on_ = prof;
        throw;
    }
    P_.dstep = nullptr;
    ff_n0_ = n0;
    prof_on_ = prof;
    graph_launches_ = launches_ - l0;
    launches_ = l0;
    AEM_CUDA(cudaStreamEndCapture(stream_, &graph));
    cudaError_t e = cudaGraphInstantiate(&graph_, graph, 0);
    cudaGraphDestroy(graph);
    AEM_CUDA(e);
    graph_g_ = g;
}

void Solver::run_graph(int n, int g) {
    Solver* self = this;
    run_batch(&self, 1, n, g);
}

// Checkpoint file: "AEMCKPT1", then int64 fields (kmax, cells, steps,
// done, far-field batch start, buffer count), the byte size of every
// setup-time device buffer, then the buffers' bytes in allocation order.
// The buffers hold the fields, CPML psi, port lines, far-field bins and
// difference buffers, per-step taps and spectra, and the constant tables;
// a handle made from the same deck allocates the same buffers in the same
// order and sizes, which the load checks.  On the fused path the field
// buffers swap every step, so the loading handle swaps its pointers when
// its step count and the snapshot's differ in parity.
namespace {
constexpr char CKPT_MAGIC[8] = {'A', 'E', 'M', 'C', 'K', 'P', 'T', '1'};
constexpr size_t CKPT_CHUNK = 64u << 20;
}  // namespace

void Solver::checkpoint_save(const std::string& path) {
    if (full_.f[0]) throw std::invalid_argument("checkpoints are not supported while the full-field export is on");
    AEM_CUDA(cudaStreamSynchronize(stream_));
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::invalid_argument("cannot write checkpoint '" + path + "'");
    void* stage = nullptr;
    bool ok = true;
    try {
        AEM_CUDA(cudaMallocHost(&stage, CKPT_CHUNK));
        const long long hdr[6] = {m_.d.kmax ? 1 : 0, (long long)m_.cells, m_.d.steps, done_, ff_n0_, (long long)nstate_};
        ok = std::fwrite(CKPT_MAGIC, 1, 8, f) == 8 && std::fwrite(hdr, sizeof hdr, 1, f) == 1;
        for (size_t b = 0; ok && b < nstate_; b++) {
            const long long n = (long long)buf_bytes_[b];
            ok = std::fwrite(&n, sizeof n, 1, f) == 1;
        }
        for (size_t b = 0; ok && b < nstate_; b++)
            for (size_t o = 0; ok && o < buf_bytes_[b]; o += CKPT_CHUNK) {
                const size_t n = std::min(CKPT_CHUNK, buf_bytes_[b] - o);
                AEM_CUDA(cudaMemcpyAsync(stage, (const char*)bufs_[b] + o, n, cudaMemcpyDeviceToHost, stream_));
                AEM_CUDA(cudaStreamSynchronize(stream_));
                ok = std::fwrite(stage, 1, n, f) == n;
                d2h_bytes_ += n;
            }
    } catch (...) {
        if (stage) cudaFreeHost(stage);
        std::fclose(f);
        throw;
    }
    cudaFreeHost(stage);
    if (std::fclose(f) != 0) ok = false;
    if (!ok) throw std::runtime_error("writing checkpoint '" + path + "' failed");
}

void Solver::checkpoint_load(const std::string& path) {
    if (full_.f[0]) throw std::invalid_argument("checkpoints are not supported while the full-field export is on");
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::invalid_argument("cannot open checkpoint '" + path + "'");
    void* stage = nullptr;
    long long hdr[6] = {0, 0, 0, 0, 0, 0};
    try {
        char magic[8];
        if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, CKPT_MAGIC, 8) != 0 || std::fread(hdr, sizeof hdr, 1, f) != 1)
            throw std::invalid_argument("'" + path + "' is not a checkpoint file");
        bool match = hdr[0] == (m_.d.kmax ? 1 : 0) && hdr[1] == (long long)m_.cells && hdr[2] == m_.d.steps &&
                     hdr[5] == (long long)nstate_ && hdr[3] >= 0 && hdr[3] <= m_.d.steps;
        for (size_t b = 0; match && b < nstate_; b++) {
            long long n = 0;
            if (std::fread(&n, sizeof n, 1, f) != 1) throw std::invalid_argument("checkpoint '" + path + "' is truncated");
            match = n == (long long)buf_bytes_[b];
        }
        if (!match) throw std::invalid_argument("checkpoint '" + path + "' was not written by a run of this deck");
        // the whole payload must be there before any buffer is overwritten,
        // so that a truncated file leaves the handle as it was
        const long pos = std::ftell(f);
        long long need = 0;
        for (size_t b = 0; b < nstate_; b++) need += (long long)buf_bytes_[b];
        if (pos < 0 || std::fseek(f, 0, SEEK_END) != 0 || (long long)std::ftell(f) - pos < need ||
            std::fseek(f, pos, SEEK_SET) != 0)
            throw std::invalid_argument("checkpoint '" + path + "' is truncated");
        AEM_CUDA(cudaStreamSynchronize(stream_));
        release_graph();
        AEM_CUDA(cudaMallocHost(&stage, CKPT_CHUNK));
        for (size_t b = 0; b < nstate_; b++)
            for (size_t o = 0; o < buf_bytes_[b]; o += CKPT_CHUNK) {
                const size_t n = std::min(CKPT_CHUNK, buf_bytes_[b] - o);
                if (std::fread(stage, 1, n, f) != n) throw std::invalid_argument("checkpoint '" + path + "' is truncated");
                AEM_CUDA(cudaMemcpyAsync((char*)bufs_[b] + o, stage, n, cudaMemcpyHostToDevice, stream_));
                AEM_CUDA(cudaStreamSynchronize(stream_));
                h2d_bytes_ += n;
            }
    } catch (...) {
        if (stage) cudaFreeHost(stage);
        std::fclose(f);
        throw;
    }
    cudaFreeHost(stage);
    std::fclose(f);
    if (fused_ && ((done_ ^ (int)hdr[3]) & 1)) {  // the same pointer swaps as one step()
        for (int c = 0; c < 3; c++) {
            std::swap(P_.E[c], P_.E2[c]);
            std::swap(P_.H[c], P_.H2[c]);
            for (int a = 0; a < 3; a++)
                for (int s = 0; s < 2; s++) std::swap(P_.psi_h[c][a][s], P_.psi_h2[c][a][s]);
        }
    }
    done_ = (int)hdr[3];
    ff_n0_ = (int)hdr[4];
}

void Solver::run_batch(Solver* const* s, int count, int n, int g) {
    std::vector<int> left(count);
    for (int i = 0; i < count; i++) {
        Solver& v = *s[i];
        left[i] = std::max(0, std::min(n, v.m_.d.steps - v.done_));
        left[i] -= v.autotune_pending(left[i]);
        // eager steps until a chunk can start (at most one far-field batch)
        while (left[i] > 0 && !v.graph_ready(g) && (v.done_ == 0 || left[i] < g || v.FF_.tb > 1 && v.ff_n0_ != v.done_ + 1)) {
            v.run(1);
            left[i]--;
        }
        if (left[i] >= g && v.graph_ready(g)) {
            if (!v.graph_ || v.graph_g_ != g) v.capture_graph(g);
            const int next = v.done_ + 1;
            AEM_CUDA(cudaMemcpyAsync(v.dstep_, &next, sizeof next, cudaMemcpyHostToDevice, v.stream_));
            v.h2d_bytes_ += sizeof next;
        }
    }
    // whole chunks, round-robin over the solvers
    for (bool any = true; any;) {
        any = false;
        for (int i = 0; i < count; i++) {
            Solver& v = *s[i];
            if (!v.graph_ || left[i] < g || v.done_ + g > v.m_.d.steps) continue;
            AEM_CUDA(cudaGraphLaunch(v.graph_, v.stream_));
            v.done_ += g;
            left[i] -= g;
            v.launches_ += v.graph_launches_;
            if (v.FF_.tb > 1) v.ff_n0_ = v.done_ + 1;
            any = true;
            // a chunk that passed a watchdog step is checked at its end
            const int K = v.m_.d.ext_watchdog;
            if (K > 0 && v.done_ / K != (v.done_ - g) / K) v.watchdog_check();
        }
    }
    // the rest eagerly (run() also bins the last far-field batch)
    for (int i = 0; i < count; i++) {
        Solver& v = *s[i];
        if (left[i] > 0 || v.done_ == v.m_.d.steps) v.run(left[i]);
    }
}

}  // namespace aem
