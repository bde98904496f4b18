// aem_deck.cpp -- inputs.txt reader and derived run parameters.
//
// Reads the positional grammar of main_fdtd/fdtd_solver.f90:726-1298 with
// Fortran list-directed semantics (every READ starts a new record, takes as
// many comma/blank separated values as it needs and drops the rest of its
// last record).  Derived quantities follow :1305-1812 in FP32 with the
// reference's operation order, so the coefficients fed to the kernels equal
// the reference's.
#include "aem_deck.h"
#include "aem_types.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace aem {
namespace {

struct Reader {
    std::vector<std::string> lines;
    size_t cur = 0;

    explicit Reader(const std::string& text) {
        std::string s;
        std::istringstream is(text);
        while (std::getline(is, s)) {
            if (!s.empty() && s.back() == '\r') s.pop_back();
            lines.push_back(s);
        }
    }
    std::vector<std::string> tokens(int n) {
        std::vector<std::string> out;
        while ((int)out.size() < n) {
            if (cur >= lines.size()) throw DeckError("unexpected end of the input file");
            const std::string& s = lines[cur++];
            size_t p = 0;
            while (p < s.size() && (int)out.size() < n) {
                while (p < s.size() && (s[p] == ' ' || s[p] == '\t')) p++;
                if (p >= s.size()) break;
                if (s[p] == ',') { p++; continue; }
                std::string t;
                if (s[p] == '\'' || s[p] == '"') {
                    char q = s[p++];
                    while (p < s.size() && s[p] != q) t += s[p++];
                    if (p < s.size()) p++;
                } else {
                    while (p < s.size() && s[p] != ',' && s[p] != ' ' && s[p] != '\t') t += s[p++];
                }
                out.push_back(t);
            }
        }
        return out;
    }
    int geti() {
        auto t = tokens(1)[0];
        char* e = nullptr;
        long v = std::strtol(t.c_str(), &e, 10);
        if (*e) throw DeckError("bad integer '" + t + "' in input file");
        return (int)v;
    }
    void geti(int n, int* o) {
        auto t = tokens(n);
        for (int q = 0; q < n; q++) {
            char* e = nullptr;
            long v = std::strtol(t[q].c_str(), &e, 10);
            if (*e) throw DeckError("bad integer '" + t[q] + "' in input file");
            o[q] = (int)v;
        }
    }
    static float tof(std::string t) {
        for (auto& c : t) if (c == 'd' || c == 'D') c = 'E';
        char* e = nullptr;
        float v = std::strtof(t.c_str(), &e);
        if (e == t.c_str()) throw DeckError("bad real '" + t + "' in input file");
        return v;
    }
    float getf() { return tof(tokens(1)[0]); }
    void getf(int n, float* o) {
        auto t = tokens(n);
        for (int q = 0; q < n; q++) o[q] = tof(t[q]);
    }
    // character(len=L) list-directed value
    std::string gets(size_t L) {
        auto t = tokens(1)[0];
        if (t.size() > L) t.resize(L);
        return t;
    }
    // read(1,'(a)') into character(len=L), adjustl(trim())
    std::string getline_trim(size_t L) {
        if (cur >= lines.size()) throw DeckError("unexpected end of the input file");
        std::string s = lines[cur++];
        if (s.size() > L) s.resize(L);
        size_t a = s.find_first_not_of(" \t"), b = s.find_last_not_of(" \t");
        return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
    }
};

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t"), b = s.find_last_not_of(" \t");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

}  // namespace

Deck parse_deck(const std::string& text, bool kmax) {
    Deck d;
    d.kmax = kmax;
    Reader r(text);
    int v3[3];
    float f3[3];
    r.geti(3, v3); d.nx = v3[0]; d.ny = v3[1]; d.nz = v3[2];
    r.getf(3, f3); d.dx = f3[0]; d.dy = f3[1]; d.dz = f3[2];
    d.steps = r.geti();
    d.factor = r.getf();
    d.f_center = r.getf();
    d.pulse_type = r.geti();
    r.geti(6, d.bc);
    for (int a = 0; a < 3; a++) d.pbc[a] = (d.bc[2 * a] == 1 && d.bc[2 * a + 1] == 1) ? 1 : 0;
    if (trim(r.gets(5)) == "IGP") {
        d.is_mirror = 1;
        std::string mt = r.gets(2);
        const char* names[6] = {"-x", "+x", "-y", "+y", "-z", "+z"};
        for (int q = 0; q < 6; q++) if (mt == names[q]) d.mirror_type = q + 1;
        d.mirror_height = r.geti();
    }
    d.excitation = r.getline_trim(15);
    if (!kmax) {
        if (d.excitation == "plane wave") {
            r.getf(2, f3); d.pw_amp = f3[0]; d.pw_delay = f3[1];
            r.getf(3, f3); d.theta = f3[0]; d.phi = f3[1]; d.pol = f3[2];
            if (d.mirror_type == 1 || d.mirror_type == 2) { d.theta_m = d.theta; d.phi_m = 180.0f - d.phi; }
            if (d.mirror_type == 3 || d.mirror_type == 4) { d.theta_m = d.theta; d.phi_m = 360.0f - d.phi; }
            if (d.mirror_type == 5 || d.mirror_type == 6) { d.theta_m = 180.0f - d.theta; d.phi_m = d.phi; }
        } else if (d.excitation == "antenna") {
            r.getf(2, f3); d.ant_amp = f3[0]; d.ant_delay = f3[1];
            d.exc_port = r.geti();
            if (d.exc_port == 0) { d.ant_amp = 0; d.ant_delay = 0; }
        }
        int np = d.pbc[0] + d.pbc[1] + d.pbc[2];
        if (np == 3) std::printf(" WARNING: ONLY PBC WALLS DETECTED - ONLY ANTENNA SOURCES CAN BE GENERATED - ONLY OUTPUT FIELDS ARE USEFUL\n");
        if (np == 2 && d.is_mirror == 1)
            throw DeckError("ERROR: USER ADDED AN IGP CONDITION TO A UNIT CELL W/ 2 SETS OF PBC - THIS IS NOT NEEDED AND INVALID");
        const char* obl = "ERROR: INCIDENT PLANE WAVE W/ OBLIQUE ANGLE W/ RESPECT TO PBC DETECTED - USE KMAX";
        if (d.pbc[0] == 1 && d.pw_amp > 0 && std::fmod(d.theta, 180.0f) != 0.0f && std::fmod(d.phi, 180.0f) != 90.0f) throw DeckError(obl);
        if (d.pbc[1] == 1 && d.pw_amp > 0 && std::fmod(d.theta, 180.0f) != 0.0f && std::fmod(d.phi, 180.0f) != 0.0f) throw DeckError(obl);
        if (d.pbc[2] == 1 && d.pw_amp > 0 && std::fmod(d.theta, 180.0f) != 90.0f) throw DeckError(obl);
    } else {
        if (d.excitation == "plane wave") {
            r.getf(2, f3); d.pw_amp = f3[0]; d.pw_delay = f3[1];
            std::string mt = trim(r.gets(5));
            std::string kd = trim(r.gets(2));
            if (kd == "-") d.k_direction = 0;
            else if (kd == "+") d.k_direction = 1;
            else throw DeckError("ERROR: INVALID PROPOGATION DIRECTION DETECTED");
            if (mt == "TE") d.mode_type = 0;
            if (mt == "TM") d.mode_type = 1;
        } else if (d.excitation == "antenna") {
            r.getf(2, f3); d.ant_amp = f3[0]; d.ant_delay = f3[1];
            d.exc_port = r.geti();
            if (d.exc_port == 0) { d.ant_amp = 0; d.ant_delay = 0; }
        }
        float k2[2];
        if (d.pbc[1] + d.pbc[2] == 2) { r.getf(2, k2); d.kc[1] = k2[0]; d.kc[2] = k2[1]; }
        else if (d.pbc[0] + d.pbc[2] == 2) { r.getf(2, k2); d.kc[0] = k2[0]; d.kc[2] = k2[1]; }
        else if (d.pbc[0] + d.pbc[1] == 2) { r.getf(2, k2); d.kc[0] = k2[0]; d.kc[1] = k2[1]; }
        int np = d.pbc[0] + d.pbc[1] + d.pbc[2];
        if (np == 3) std::printf(" WARNING: ONLY PBC WALLS DETECTED - ONLY ANTENNA SOURCES CAN BE GENERATED - ONLY OUTPUT FIELDS ARE USEFUL\n");
        if (np == 2 && d.is_mirror == 1)
            throw DeckError("ERROR: USER ADDED AN IGP CONDITION TO A UNIT CELL W/ 2 SETS OF PBC - THIS IS NOT NEEDED AND INVALID");
        if (np == 1) throw DeckError("ERROR: USER ONLY ADDED 1 PBC W/ KMAX - THIS IS INVALID");
    }
    const float pi = 3.14159265358979323846f;
    d.n_ff = r.geti();
    if (d.n_ff > 0) { r.geti(3, v3); d.ic = v3[0]; d.jc = v3[1]; d.kc_ = v3[2]; }
    for (int q = 0; q < d.n_ff; q++) {
        r.getf(2, f3);
        d.ff_theta.push_back(pi / 180.0f * f3[0]);
        d.ff_phi.push_back(pi / 180.0f * f3[1]);
    }
    if (trim(r.gets(10)) == "yes") {
        d.video_on = 1;
        std::string s = trim(r.gets(3));
        if (s == "x") d.slice_dir = 0;
        if (s == "y") d.slice_dir = 1;
        if (s == "z") d.slice_dir = 2;
        d.slice_loc = r.geti();
    }
    d.export_all = trim(r.gets(5));
    d.filename = trim(r.gets(30));
    int ntot = r.geti();
    for (int q = 0; q < ntot; q++) {
        std::string mt = trim(r.gets(30));
        if (mt == "volume") {
            VolumeMaterial m;
            std::string kind = trim(r.gets(7));
            m.id = r.getf();
            r.getf(3, m.eps);
            r.getf(3, m.sig);
            if (kind == "plasma") {
                m.npoles = r.geti();
                if (m.npoles > 6) throw DeckError("ERROR: AT MOST 6 POLES PER MATERIAL ARE SUPPORTED");
                for (int p = 0; p < m.npoles; p++) { r.getf(3, m.wp[p]); r.getf(3, m.gam[p]); }
            }
            d.mats.push_back(m);
        } else if (mt == "sheet") {
            SheetMaterial s;
            s.id = r.getf();
            float imped = r.getf();
            float mn = d.dx;
            if (d.dy < mn) mn = d.dy;
            if (d.dz < mn) mn = d.dz;
            d.sheet_thickness = mn / 5000.0f;  // ref :957
            for (int a = 0; a < 3; a++) {
                s.ep[a] = 1.0f;
                s.sig[a] = imped == 0 ? 1E20f : 1.0f / (imped * d.sheet_thickness);
            }
            d.smats.push_back(s);
        }
    }
    if (trim(r.gets(5)) == "yes") d.bulk_file = trim(r.gets(50));
    int nobj = r.geti();
    for (int q = 0; q < nobj; q++) {
        std::string ot = trim(r.gets(15));
        Object o;
        if (ot == "block") {
            o.kind = Object::Block;
            o.mat = r.geti();
            r.geti(3, o.a);
            r.geti(3, o.b);
        } else if (ot == "sphere") {
            o.kind = Object::Sphere;
            o.mat = r.geti();
            r.geti(3, o.a);
            o.b[0] = r.geti();
        } else if (ot == "cylinder") {
            o.kind = Object::Cylinder;
            o.mat = r.geti();
            std::string ax = trim(r.gets(3));
            o.axis = ax == "x" ? 0 : ax == "y" ? 1 : ax == "z" ? 2 : -1;
            r.geti(3, o.a);
            int v2[2];
            r.geti(2, v2);
            o.b[0] = v2[0]; o.b[1] = v2[1];
        } else {
            continue;  // the reference silently ignores unknown object kinds
        }
        d.objects.push_back(o);
    }
    int nsh = r.geti();
    for (int q = 0; q < nsh; q++) {
        std::string sp = trim(r.gets(3));
        int n = sp == "x" ? 0 : sp == "y" ? 1 : sp == "z" ? 2 : -1;
        if (n < 0) continue;
        Sheet s;
        s.normal = n;
        s.mat = r.geti();
        s.pos = r.geti();
        r.geti(2, s.start);
        r.geti(2, s.len);
        d.sheets.push_back(s);
    }
    int npt = r.geti();
    for (int q = 0; q < npt; q++) {
        std::string pt = trim(r.gets(7));
        Port p;
        const float c0 = 299792458.0f;
        if (pt == "basic") {
            std::string cp = trim(r.gets(3));
            p.dir = cp == "x" ? 0 : cp == "y" ? 1 : 2;
            float z0 = r.getf();
            p.L = z0 / c0;
            p.C = 1.0f / (z0 * c0);
            r.getf(3, p.loc);
            if (p.loc[0] == 1 || p.loc[1] == 1 || p.loc[2] == 1)
                throw DeckError("ERROR: FDTD SOFTWARE DOES NOT CURRENTLY SUPPORT PLACING AN INTERNAL LUMPED PORT AT A FIRST CUBE");
            r.getf(3, p.size);
            for (int a = 0; a < 3; a++) if (a != p.dir) p.size[a] += 1.0f;
        } else if (pt == "gridded") {
            p.gridded = 1;
            std::string cp = trim(r.gets(3));
            const char* names[6] = {"-x", "+x", "-y", "+y", "-z", "+z"};
            for (int s = 0; s < 6; s++) if (cp == names[s]) { p.dir = s / 2; p.side = s; }
            float z0 = r.getf();
            p.L = z0 / c0;
            p.C = 1.0f / (z0 * c0);
            r.getf(3, p.loc);
            if (p.loc[0] == 1 || p.loc[1] == 1 || p.loc[2] == 1)
                throw DeckError("ERROR: FDTD SOFTWARE DOES NOT CURRENTLY SUPPORT PLACING AN INTERNAL LUMPED PORT AT A FIRST CUBE");
            r.getf(2, p.size);
            p.feed = trim(r.gets(30));
        } else {
            continue;
        }
        d.ports.push_back(p);
    }
    d.num_spice_ports = r.geti();
    return d;
}

Deck parse_deck_file(const std::string& path, bool kmax) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw DeckError("cannot open input file '" + path + "'");
    std::stringstream ss;
    ss << f.rdbuf();
    Deck d = parse_deck(ss.str(), kmax);
    // optional sidecar with run extensions
    std::ifstream x(path + ".b200", std::ios::binary);
    if (x) {
        std::stringstream xs;
        xs << x.rdbuf();
        apply_extensions(d, xs.str());
    }
    return d;
}

void apply_extensions(Deck& d, const std::string& text) {
    std::istringstream x(text);
    std::string line;
    while (std::getline(x, line)) {
        std::istringstream ls(line);
        std::string key, val;
        if (!(ls >> key) || key[0] == '#') continue;
        if (!(ls >> val)) throw DeckError("extension '" + key + "' needs a value");
        if (key == "pml_cells") {
            char* end = nullptr;
            long v = std::strtol(val.c_str(), &end, 10);
            if (*end || v < 0 || v > AEM_MAX_PML - 2) throw DeckError("extension pml_cells must be 0.." + std::to_string(AEM_MAX_PML - 2));
            d.ext_pml_cells = (int)v;
        } else if (key == "geometry_bin") {
            if (val != "yes" && val != "no") throw DeckError("extension geometry_bin must be yes or no");
            d.ext_geometry_bin = val == "yes";
        } else if (key == "watchdog") {
            // watchdog K: every K steps, stop the run if E or H holds a
            // non-finite value
            char* end = nullptr;
            long v = std::strtol(val.c_str(), &end, 10);
            if (*end || v < 0 || v > 1000000000L) throw DeckError("extension watchdog must be a step count >= 0");
            d.ext_watchdog = (int)v;
        } else if (key == "dft_freqs") {
            // dft_freqs f_start f_stop count: count frequencies spaced evenly
            // from f_start to f_stop inclusive (Hz)
            std::string v1, v2;
            char *e0 = nullptr, *e1 = nullptr, *e2 = nullptr;
            if (!(ls >> v1 >> v2)) throw DeckError("extension dft_freqs needs f_start f_stop count");
            const double f0 = std::strtod(val.c_str(), &e0), f1 = std::strtod(v1.c_str(), &e1);
            const long n = std::strtol(v2.c_str(), &e2, 10);
            if (*e0 || *e1 || *e2 || !(f0 >= 0.0) || !(f1 >= f0) || n < 1 || n > AEM_MAX_DFT_FREQS)
                throw DeckError("extension dft_freqs needs 0 <= f_start <= f_stop and 1 <= count <= " +
                                std::to_string(AEM_MAX_DFT_FREQS));
            d.ext_dft_freqs.resize((size_t)n);
            for (long q = 0; q < n; q++) d.ext_dft_freqs[q] = n == 1 ? f0 : f0 + (f1 - f0) * (double)q / (double)(n - 1);
        } else if (key == "cpml_grading") {
            // cpml_grading m sigma_factor kappa_max alpha_max
            std::string v1, v2, v3;
            char *e0 = nullptr, *e1 = nullptr, *e2 = nullptr, *e3 = nullptr;
            if (!(ls >> v1 >> v2 >> v3)) throw DeckError("extension cpml_grading needs m sigma_factor kappa_max alpha_max");
            const long m = std::strtol(val.c_str(), &e0, 10);
            const float sf = std::strtof(v1.c_str(), &e1), km = std::strtof(v2.c_str(), &e2), am = std::strtof(v3.c_str(), &e3);
            if (*e0 || *e1 || *e2 || *e3 || m < 1 || m > 8 || !(sf >= 0.0f) || !(km >= 1.0f) || !(am >= 0.0f))
                throw DeckError("extension cpml_grading needs 1 <= m <= 8, sigma_factor >= 0, kappa_max >= 1, alpha_max >= 0");
            d.ext_cpml = true;
            d.ext_cpml_m = (int)m;
            d.ext_cpml_sigma = sf;
            d.ext_cpml_kappa = km;
            d.ext_cpml_alpha = am;
        } else if (key == "coef_precision") {
            // coef_precision 32 (reference FP32 arithmetic) or 64 (the
            // material and CPML tables in FP64 on the GPU)
            if (val != "32" && val != "64") throw DeckError("extension coef_precision must be 32 or 64");
            d.ext_coef64 = val == "64";
        } else if (key == "autotune") {
            // autotune N: at the first step, time candidate launch shapes of
            // the two-kernel update for N steps each (8 candidates)
            char* end = nullptr;
            long v = std::strtol(val.c_str(), &end, 10);
            if (*end || v < 0 || v > 1000) throw DeckError("extension autotune must be 0..1000 steps per candidate");
            d.ext_autotune = (int)v;
        } else if (key == "tfsf_inset") {
            char* end = nullptr;
            long v = std::strtol(val.c_str(), &end, 10);
            if (*end || v < 2 || v > 1000000L) throw DeckError("extension tfsf_inset must be a cell index >= 2");
            d.ext_tfsf_inset = (int)v;
        } else if (key == "probe") {
            // probe i j k: reference cell indices, 1 <= i <= nx - 1 (the
            // cell-centred average reads i and i+1)
            std::string v1, v2;
            char *e0 = nullptr, *e1 = nullptr, *e2 = nullptr;
            if (!(ls >> v1 >> v2)) throw DeckError("extension probe needs i j k");
            const long i = std::strtol(val.c_str(), &e0, 10), j = std::strtol(v1.c_str(), &e1, 10),
                       k = std::strtol(v2.c_str(), &e2, 10);
            if (*e0 || *e1 || *e2 || i < 1 || j < 1 || k < 1) throw DeckError("extension probe needs cell indices >= 1");
            if ((int)d.ext_probes.size() >= AEM_MAX_PROBES)
                throw DeckError("extension probe: at most " + std::to_string(AEM_MAX_PROBES) + " probes");
            d.ext_probes.push_back({(int)i, (int)j, (int)k});
        } else {
            throw DeckError("unknown extension '" + key + "'");
        }
    }
}

// ref :1305-1812 (FP32, same operation order as the reference)
void derive(Deck& d) {
    const float c0 = 299792458.0f, mu0 = 1.25663706E-6f, ep0 = 8.85418782E-12f, pi = 3.14159265358979323846f;
    const float dx = d.dx, dy = d.dy, dz = d.dz;
    d.del_t = 0.98f / (c0 * std::pow(1.0f / (dx * dx) + 1.0f / (dy * dy) + 1.0f / (dz * dz), 0.5f)) / d.factor;
    d.X = d.nx + 1 + d.pbc[0];
    d.Y = d.ny + 1 + d.pbc[1];
    d.Z = d.nz + 1 + d.pbc[2];
    const float sumL = dx * (float)d.X + dy * (float)d.Y + dz * (float)d.Z;
    d.r_relay = 1.0f;
    if (sumL > d.r_relay) d.r_relay = sumL * 2.0f;
    d.len_ff = (int)((float)d.steps + (d.r_relay + sumL) / (c0 * d.del_t));
    float mind = dx;
    if (dy < mind) mind = dy;
    if (dz < mind) mind = dz;
    d.port_array_size = (int)((float)d.steps * d.del_t * c0 / mind / 2.0f + 100.0f);
    int pml = d.ext_pml_cells > 0 ? d.ext_pml_cells + 1 : 11;
    for (int a = 0; a < 3; a++) {
        d.npml[a][0] = d.npml[a][1] = d.pbc[a] ? 0 : pml;
    }
    const int N[3] = {d.X, d.Y, d.Z};
    if (d.slice_dir == 0) { d.vid1 = d.Y - 1 - d.pbc[1]; d.vid2 = d.Z - 1 - d.pbc[2]; }
    if (d.slice_dir == 1) { d.vid1 = d.X - 1 - d.pbc[0]; d.vid2 = d.Z - 1 - d.pbc[2]; }
    if (d.slice_dir == 2) { d.vid1 = d.X - 1 - d.pbc[0]; d.vid2 = d.Y - 1 - d.pbc[1]; }
    float th = pi / 180.0f * d.theta, ph = pi / 180.0f * d.phi, po = pi / 180.0f * d.pol;
    float thm = pi / 180.0f * d.theta_m, phm = pi / 180.0f * d.phi_m;
    d.theta = th; d.phi = ph; d.pol = po; d.theta_m = thm; d.phi_m = phm;
    for (int a = 0; a < 3; a++) {
        d.lo[a] = 1;
        d.hi[a] = N[a] - 1;
        if (!d.pbc[a]) { d.lo[a] = d.npml[a][0] + 3; d.hi[a] = N[a] - d.npml[a][1] - 3; }
        // extension tfsf_inset: the TF/SF planes (and the far-field box
        // derived from them) at index N and X - N instead of npml + 3
        if (!d.pbc[a] && d.ext_tfsf_inset > 0) {
            if (d.ext_tfsf_inset <= d.npml[a][0] || N[a] - d.ext_tfsf_inset >= N[a] - d.npml[a][1] ||
                N[a] - d.ext_tfsf_inset <= d.ext_tfsf_inset)
                throw DeckError("extension tfsf_inset: the TF/SF box must lie between the CPML slabs");
            d.lo[a] = d.ext_tfsf_inset;
            d.hi[a] = N[a] - d.ext_tfsf_inset;
        }
    }
    if (d.is_mirror) {  // ref :1402-1447
        int a = (d.mirror_type - 1) / 2;
        if (d.mirror_type % 2 == 1) {
            d.lo[a] = d.mirror_height + 1; d.wall_lo[a] = 0; d.mir_off[a] = 2.0f * (float)d.lo[a];
            d.npml[a][0] = 1; d.use_mir[a] = 1;
        } else {
            d.hi[a] = d.mirror_height; d.wall_hi[a] = 0; d.mir_off[a] = 2.0f * (float)d.hi[a];
            d.npml[a][1] = 0; d.use_mir[a] = 1;
        }
    }
    // plane-wave delay lookup, ref :1451-1494 and :1522-1565
    auto lookup = [&](float t, float p, int* del) {
        if (t >= 0.0f && t <= pi / 2.0f) {
            if (p >= 0.0f && p <= pi / 2.0f) { del[0] = d.lo[0]; del[1] = d.lo[1]; del[2] = d.lo[2]; }
            if (p > pi / 2.0f && p <= pi) { del[0] = d.hi[0]; del[1] = d.lo[1]; del[2] = d.lo[2]; }
            if (p > pi && p <= 3.0f * pi / 2.0f) { del[0] = d.hi[0]; del[1] = d.hi[1]; del[2] = d.lo[2]; }
            if (p > 3.0f * pi / 2.0f && p < 2.0f * pi) { del[0] = d.lo[0]; del[1] = d.hi[1]; del[2] = d.lo[2]; }
        }
        if (t > pi / 2.0f && t <= pi) {
            if (p >= 0.0f && p <= pi / 2.0f) { del[0] = d.lo[0]; del[1] = d.lo[1]; del[2] = d.hi[2]; }
            if (p > pi / 2.0f && p <= pi) { del[0] = d.hi[0]; del[1] = d.lo[1]; del[2] = d.hi[2]; }
            if (p > pi && p <= 3.0f * pi / 2.0f) { del[0] = d.hi[0]; del[1] = d.hi[1]; del[2] = d.hi[2]; }
            if (p > 3.0f * pi / 2.0f && p < 2.0f * pi) { del[0] = d.lo[0]; del[1] = d.hi[1]; del[2] = d.hi[2]; }
        }
    };
    lookup(th, ph, d.delay);
    if (!d.kmax) {  // ref :1499-1504
        float s = std::sqrt(ep0 / mu0);
        d.WH[0] = d.pw_amp * (std::sin(po) * std::sin(ph) + std::cos(po) * std::cos(th) * std::cos(ph)) * s;
        d.WH[1] = d.pw_amp * (-1.0f * std::sin(po) * std::cos(ph) + std::cos(po) * std::cos(th) * std::sin(ph)) * s;
        d.WH[2] = d.pw_amp * (-1.0f * std::cos(po) * std::sin(th)) * s;
        d.WE[0] = d.pw_amp * (std::cos(po) * std::sin(ph) - std::sin(po) * std::cos(th) * std::cos(ph));
        d.WE[1] = d.pw_amp * (-1.0f * std::cos(po) * std::cos(ph) - std::sin(po) * std::cos(th) * std::sin(ph));
        d.WE[2] = d.pw_amp * (std::sin(po) * std::sin(th));
    } else {  // ref :1507-1517
        if (d.mode_type == 0) for (int a = 0; a < 3; a++) d.WE[a] = 2.0f * d.pw_amp;
        if (d.mode_type == 1) for (int a = 0; a < 3; a++) d.WH[a] = 2.0f * std::sqrt(ep0 / mu0) * d.pw_amp;
    }
    lookup(thm, phm, d.delay_m);
    if (d.is_mirror) {  // ref :1571-1635
        int a = (d.mirror_type - 1) / 2;
        if (d.mirror_type % 2 == 1) d.delay_m[a] = d.mirror_height + (d.mirror_height - d.hi[a]);
        else d.delay_m[a] = d.mirror_height + (d.mirror_height - d.lo[a]);
        for (int c = 0; c < 3; c++) {
            float sE = (c == a) ? 1.0f : -1.0f;  // tangential E flips, normal E kept
            d.WE_m[c] = sE == 1.0f ? d.WE[c] : -1.0f * d.WE[c];
            d.WH_m[c] = (c == a) ? -1.0f * d.WH[c] : d.WH[c];
            if (c != a) d.J_mir[c] = -1.0f;
        }
        d.M_mir[a] = -1.0f;
    }
    // far-field box, ref :1638-1680
    for (int a = 0; a < 3; a++) { d.ff_lo[a] = d.lo[a] - 2; d.ff_hi[a] = d.hi[a] + 1; }
    if (d.is_mirror) {
        int a = (d.mirror_type - 1) / 2;
        if (d.mirror_type % 2 == 1) d.ff_lo[a] = d.lo[a] + 1;
        else d.ff_hi[a] = d.hi[a] - 2;
    }
    for (int a = 0; a < 3; a++) if (d.pbc[a]) { d.ff_lo[a] = 1; d.ff_hi[a] = N[a] - 2; }
    // CPML maxima, ref :1685-1706
    float eta = std::pow(mu0 / ep0 * 1.0f, 0.5f);
    float lg = -1.0f * std::log(1.0E-6f);
    const float dl[3] = {dx, dy, dz};
    float sfac = d.kmax ? 1.25f : 1.0f;
    for (int a = 0; a < 3; a++) d.sig_max[a] = lg * ((float)(3 + 1) / (dl[a] * eta)) / (float)(2 * d.npml[a][0]) * sfac;
    if (!d.kmax) d.alpha_max = 0.03f;
    else d.alpha_max = 0.03f + 0.9f * (std::sqrt(d.kc[1] * d.kc[1] + d.kc[2] * d.kc[2] + d.kc[0] * d.kc[0])) / 377.0f;
    d.kappa_max = 7.0f;
    d.cpml_m = 3;
    if (d.ext_cpml) {
        // extension cpml_grading: sigma_max = sigma_factor (m+1) / (eta0 d)
        d.cpml_m = d.ext_cpml_m;
        for (int a = 0; a < 3; a++) d.sig_max[a] = d.ext_cpml_sigma * ((float)(d.cpml_m + 1) / (dl[a] * eta));
        d.alpha_max = d.ext_cpml_alpha;
        d.kappa_max = d.ext_cpml_kappa;
    }
    // pulse, ref :1710-1725
    if (!d.kmax) {
        d.spread = 1.0f / (2.0f * pi * d.f_center);
        if (d.pulse_type == 1) d.t_spread = 5.0f * d.spread + d.pw_delay + d.ant_delay;
        if (d.pulse_type == 2) d.t_spread = 6.0f * d.spread + d.pw_delay + d.ant_delay;
    } else {
        d.spread = 4.0f / (2.0f * pi * d.f_center);
        d.t_spread = 5.0f * d.spread + d.pw_delay + d.ant_delay;
        d.f_adj = (std::sqrt(d.kc[1] * d.kc[1] + d.kc[2] * d.kc[2] + d.kc[0] * d.kc[0]) * c0) / (2.0f * pi) + d.f_center;
        // plane and polarisation selectors, ref :1729-1806
        for (int a = 0; a < 3; a++) {
            int b = (a + 1) % 3, c = (a + 2) % 3;
            if (!(d.pbc[b] && d.pbc[c])) continue;
            if (d.k_direction == 1) { d.k_pl_H = d.lo[a] - 1; d.k_pl_E = d.lo[a]; }
            else { d.k_pl_H = d.hi[a]; d.k_pl_E = d.hi[a]; }
            int u = b < c ? b : c, v = b < c ? c : b;  // (y,z), (x,z), (x,y)
            float ku = d.kc[u], kv = d.kc[v];
            float n = std::sqrt(kv * kv + ku * ku);
            if (ku == 0 && kv != 0) { d.knum[u] = 0; d.knum[v] = kv / n; }
            if (ku != 0 && kv == 0) { d.knum[u] = ku / n; d.knum[v] = 0; }
            if (ku == 0 && kv == 0) { d.knum[u] = 0; d.knum[v] = 1; }
            if (ku != 0 && kv != 0) { d.knum[u] = ku / n; d.knum[v] = kv / n; }
        }
    }
    float a1 = std::sin(th) * std::cos(ph) * (float)d.X * dx;
    float a2 = std::sin(th) * std::sin(ph) * (float)d.Y * dy;
    float a3 = std::cos(th) * (float)d.Z * dz;
    d.min_steps = 2.0f * d.t_spread / d.del_t + std::sqrt(a1 * a1 + a2 * a2 + a3 * a3) / (c0 * d.del_t);
}

}  // namespace aem
