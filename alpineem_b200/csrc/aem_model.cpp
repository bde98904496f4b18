// aem_model.cpp -- builds the B200 data layout from a parsed deck.
//
// Restates the reference setup (main_fdtd/fdtd_solver.f90) for a layout
// of per-cell uint8 material IDs instead of full coefficient arrays:
//   rasterisation of bulk file/objects/sheets  :2051-2352
//   PBC cell fill (periodic axes stored once)  :2360-2508
//   cell->edge averaging, index-1 default      :2513-2607, :2609-2757
//   Ga/Gb and Drude Ja/Jb (FP64 intermediate)  :2832-2918
//   sheet thickness-weighted overrides         :2922-3120
//   Drude bounding boxes                       :3126-3248
//   CPML b/c, kappa and den_* tables           :3404-3666
//   gridded feeds                              :3723-3744
#include "aem_model.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <thread>

namespace aem {

namespace {

constexpr float kEp0 = 8.85418782E-12f;

std::string resolve(const std::string& dir, const std::string& f) {
    if (f.empty() || f[0] == '/' || dir.empty()) return f;
    return dir + "/" + f;
}

// Ga / Gb of the reference (:2837-2853), FP32 operation order preserved
inline float ga_of(float s, float e, float dt) {
    return (1.0f - s * dt / (2.0f * kEp0 * e)) / (1.0f + s * dt / (2.0f * kEp0 * e));
}
inline float gb_of(float s, float e, float dt) {
    return (dt / (kEp0 * e)) / (1.0f + s * dt / (2.0f * kEp0 * e));
}
// Drude coefficients (:2870-2875) -- Jb carries an FP64 intermediate
inline float ja_of(float ls, float dt) { return (1.0f - ls * dt / 2.0f) / (1.0f + ls * dt / 2.0f); }
inline float jb_of(float fr, float ls, float dt) {
    return (float)(((double)fr * (double)fr * (double)kEp0 * (double)dt / 2.0) / (double)(1.0f + ls * dt / 2.0f));
}

// The four cells averaged onto an E edge of component `c` (:2516-2527):
// Ex uses (j,k) offsets, Ey (i,k), Ez (i,j).
inline void stencil(int c, int i, int j, int k, int cell[4][3]) {
    int d[4][3] = {};
    if (c == 0) { int o[4][3] = {{0, 0, 0}, {0, -1, 0}, {0, 0, -1}, {0, -1, -1}}; memcpy(d, o, sizeof d); }
    if (c == 1) { int o[4][3] = {{0, 0, 0}, {-1, 0, 0}, {0, 0, -1}, {-1, 0, -1}}; memcpy(d, o, sizeof d); }
    if (c == 2) { int o[4][3] = {{0, 0, 0}, {-1, 0, 0}, {0, -1, 0}, {-1, -1, 0}}; memcpy(d, o, sizeof d); }
    for (int q = 0; q < 4; q++) { cell[q][0] = i + d[q][0]; cell[q][1] = j + d[q][1]; cell[q][2] = k + d[q][2]; }
}

// Sheet stencils of component c for sheets normal to n (:2537-2578): the
// reference averages in-plane cells, counting some twice.
inline void sheet_stencil(int n, int c, int i, int j, int k, int cell[4][3]) {
    int o[4][3];
    auto set = [&](int a0, int a1, int a2, int b0, int b1, int b2, int c0, int c1, int c2, int d0, int d1, int d2) {
        int t[4][3] = {{a0, a1, a2}, {b0, b1, b2}, {c0, c1, c2}, {d0, d1, d2}};
        memcpy(o, t, sizeof o);
    };
    if (n == 0) {
        if (c == 0) set(0, 0, 0, 0, -1, 0, 0, 0, -1, 0, -1, -1);
        if (c == 1) set(0, 0, 0, 0, 0, -1, 0, 0, 0, 0, 0, -1);
        if (c == 2) set(0, 0, 0, 0, -1, 0, 0, 0, 0, 0, -1, 0);
    } else if (n == 1) {
        if (c == 0) set(0, 0, 0, 0, 0, 0, 0, 0, -1, 0, 0, -1);
        if (c == 1) set(0, 0, 0, 0, 0, -1, -1, 0, 0, -1, 0, -1);
        if (c == 2) set(0, 0, 0, -1, 0, 0, 0, 0, 0, -1, 0, 0);
    } else {
        if (c == 0) set(0, 0, 0, 0, -1, 0, 0, 0, 0, 0, -1, 0);
        if (c == 1) set(0, 0, 0, -1, 0, 0, 0, 0, 0, -1, 0, 0);
        if (c == 2) set(0, 0, 0, -1, 0, 0, 0, -1, 0, -1, -1, 0);
    }
    for (int q = 0; q < 4; q++) { cell[q][0] = i + o[q][0]; cell[q][1] = j + o[q][1]; cell[q][2] = k + o[q][2]; }
}

struct SheetCells {
    // per normal: plane index -> sigma over the plane's cells [pos_b][pos_a]
    std::map<int, std::vector<float>> plane[3];
};

}  // namespace

// true when the reference leaves this edge at its vacuum default: the
// averaging loops run over 2..N-1 on every axis and only periodic axes get
// index 1 filled afterwards (:2513, :2609).
static bool edge_unaveraged(const HostModel& m, int i, int j, int k) {
    const int idx[3] = {i, j, k};
    for (int a = 0; a < 3; a++)
        if (!m.d.pbc[a] && idx[a] == 1) return true;
    return false;
}

void edge_material(const HostModel& m, int comp, int i, int j, int k, float* eps, float* sig, float* wp, float* gam) {
    if (edge_unaveraged(m, i, j, k)) {
        *eps = 1.0f; *sig = 0.0f;
        for (int p = 0; p < m.npoles; p++) { wp[p] = 0.0f; gam[p] = 0.0f; }
        return;
    }
    int cell[4][3];
    stencil(comp, i, j, k, cell);
    const AemMaterial* mm[4];
    for (int q = 0; q < 4; q++) mm[q] = &m.mats[m.cell_id[m.lin(cell[q][0], cell[q][1], cell[q][2])]];
    *eps = (mm[0]->eps[comp] + mm[1]->eps[comp] + mm[2]->eps[comp] + mm[3]->eps[comp]) / 4.0f;
    *sig = (mm[0]->sig[comp] + mm[1]->sig[comp] + mm[2]->sig[comp] + mm[3]->sig[comp]) / 4.0f;
    for (int p = 0; p < m.npoles; p++) {
        wp[p] = (mm[0]->wp[p][comp] + mm[1]->wp[p][comp] + mm[2]->wp[p][comp] + mm[3]->wp[p][comp]) / 4.0f;
        gam[p] = (mm[0]->gam[p][comp] + mm[1]->gam[p][comp] + mm[2]->gam[p][comp] + mm[3]->gam[p][comp]) / 4.0f;
    }
}

void build_model(HostModel& m, const std::string& workdir, const float* bulk, size_t bulk_n) {
    Deck& d = m.d;
    const int N[3] = {d.X, d.Y, d.Z};
    for (int a = 0; a < 3; a++) m.S[a] = d.pbc[a] ? N[a] - 2 : N[a];
    for (int a = 0; a < 3; a++)
        if (m.S[a] < 2) throw DeckError("grid too small");
    m.PX = (m.S[0] + 31) / 32 * 32;
    m.plane = (long long)m.PX * m.S[1];
    m.cells = m.plane * m.S[2];
    if (d.mats.size() + 1 > AEM_MAX_MATERIALS) throw DeckError("at most 255 volume materials are supported");

    // material table; slot 0 is the background (vacuum)
    m.npoles = 0;
    bool is_plasma = false;
    for (auto& vm : d.mats)
        if (vm.npoles > 0) { m.npoles = std::max(m.npoles, vm.npoles); is_plasma = true; }
    m.mats.assign(d.mats.size() + 1, AemMaterial{});
    for (int a = 0; a < 3; a++) { m.mats[0].eps[a] = 1.0f; m.mats[0].sig[a] = 0.0f; }
    for (size_t r = 0; r < d.mats.size(); r++) {
        AemMaterial& am = m.mats[r + 1];
        for (int a = 0; a < 3; a++) { am.eps[a] = d.mats[r].eps[a]; am.sig[a] = d.mats[r].sig[a]; }
        for (int p = 0; p < d.mats[r].npoles; p++)
            for (int a = 0; a < 3; a++) { am.wp[p][a] = d.mats[r].wp[p][a]; am.gam[p][a] = d.mats[r].gam[p][a]; }
    }
    auto find_mat = [&](float id, int prev) {
        int r0 = prev;
        for (size_t r = 0; r < d.mats.size(); r++) if (id == d.mats[r].id) r0 = (int)r + 1;
        return r0;
    };

    // geometry output (float32, (4,gx,gy,gz) column-major), ref :1963, :2355
    const int gx = N[0] - 1 - d.pbc[0], gy = N[1] - 1 - d.pbc[1], gz = N[2] - 1 - d.pbc[2];
    if (d.ext_geometry_bin) m.geometry.assign((size_t)4 * gx * gy * gz, 0.0f);
    else m.geometry.clear();
    auto geo = [&](int c, int i, int j, int k) -> float* {
        if (m.geometry.empty() || i < 1 || j < 1 || k < 1 || i > gx || j > gy || k > gz) return nullptr;
        return &m.geometry[(((size_t)(k - 1) * gy + (j - 1)) * gx + (i - 1)) * 4 + c];
    };
    // a cell write the reference keeps: inside 1..N-1 and, on periodic axes,
    // not the duplicated layer N-1 (overwritten by the PBC cell fill)
    auto cell_ok = [&](int i, int j, int k) {
        const int idx[3] = {i, j, k};
        for (int a = 0; a < 3; a++) {
            if (idx[a] < 1 || idx[a] > N[a] - 1) return false;
            if (d.pbc[a] && idx[a] == N[a] - 1) return false;
        }
        return true;
    };

    // the host reads the ids for sheet overrides, Drude boxes and the
    // geometry output; without those the device rasterises them
    // (AEM_HOST_RASTER=1 keeps the host builder, for comparison)
    const char* host_env = std::getenv("AEM_HOST_RASTER");
    m.raster_device = d.sheets.empty() && !is_plasma && !d.ext_geometry_bin && !(host_env && host_env[0] == '1');
    m.raster_bulk = nullptr;
    m.raster_file.clear();
    m.raster_map.clear();
    m.cell_id.clear();
    if (!m.raster_device) {
        m.cell_id.resize((size_t)m.cells);  // uninitialised: zeroed plane by plane in parallel
        par_for(m.S[2], [&](int z) { std::memset(m.cell_id.data() + (size_t)z * m.plane, 0, (size_t)m.plane); });
    }
    if (!d.bulk_file.empty()) {  // ref :2051-2095
        const size_t nbulk = (size_t)gx * gy * gz;
        std::vector<float> file_data;
        const float* bg = bulk;
        if (bg) {
            if (bulk_n != nbulk)
                throw DeckError("bulk geometry has " + std::to_string(bulk_n) + " values, the grid needs " + std::to_string(nbulk));
        } else {
            std::string path = resolve(workdir, d.bulk_file);
            std::ifstream f(path, std::ios::binary);
            if (!f) throw DeckError("cannot open bulk geometry file '" + path + "'");
            std::vector<float>& fd = m.raster_device ? m.raster_file : file_data;
            fd.resize(nbulk);
            f.read((char*)fd.data(), (std::streamsize)(nbulk * sizeof(float)));
            if ((size_t)f.gcount() != nbulk * sizeof(float)) throw DeckError("bulk geometry file '" + path + "' is too short");
            bg = fd.data();
        }
        int mx = 0;
        for (auto& vm : d.mats) mx = std::max(mx, (int)vm.id);
        std::vector<int> tmp((size_t)mx + 1, 0);
        for (size_t r = 0; r < d.mats.size(); r++) tmp[(int)d.mats[r].id] = (int)r + 1;
        if (m.raster_device) {
            m.raster_bulk = bg;
            m.raster_map = std::move(tmp);
        } else par_for(gz, [&](int kk) {  // planes write disjoint cells
            const int k = kk + 1;
            for (int j = 1; j <= gy; j++)
                for (int i = 1; i <= gx; i++) {
                    float v = bg[((size_t)(k - 1) * gy + (j - 1)) * gx + (i - 1)];
                    int iv = (int)v;
                    int mid = (iv >= 0 && iv <= mx) ? tmp[iv] : 0;
                    if (mid != 0) m.cell_id[m.lin(i, j, k)] = (uint8_t)mid;
                    if (float* g = geo(0, i, j, k)) *g = v;
                }
        });
    }
    int mid = 0;
    for (auto& o : d.objects) {  // ref :2101-2288
        if (m.raster_device) break;  // objects are drawn by the device, in the same order
        mid = find_mat((float)o.mat, mid);
        auto put = [&](int i, int j, int k) {
            if (cell_ok(i, j, k)) m.cell_id[m.lin(i, j, k)] = (uint8_t)mid;
            if (float* g = geo(0, i, j, k)) *g = (float)o.mat;
        };
        if (o.kind == Object::Block) {
            for (int k = o.a[2]; k <= o.a[2] + o.b[2] - 1; k++)
                for (int j = o.a[1]; j <= o.a[1] + o.b[1] - 1; j++)
                    for (int i = o.a[0]; i <= o.a[0] + o.b[0] - 1; i++) put(i, j, k);
        } else if (o.kind == Object::Sphere) {
            int r = o.b[0];
            for (int k = o.a[2] - r; k <= o.a[2] + r - 1; k++)
                for (int j = o.a[1] - r; j <= o.a[1] + r - 1; j++)
                    for (int i = o.a[0] - r; i <= o.a[0] + r - 1; i++) {
                        float x = (float)i - (float)o.a[0] + 0.5f, y = (float)j - (float)o.a[1] + 0.5f,
                              z = (float)k - (float)o.a[2] + 0.5f;
                        if ((x * x + y * y + z * z) <= (float)r * (float)r) put(i, j, k);
                    }
        } else {
            int L = o.b[0], r = o.b[1], ax = o.axis;
            if (ax < 0) continue;
            int lo[3], hi[3];
            for (int a = 0; a < 3; a++) {
                if (a == ax) { lo[a] = o.a[a]; hi[a] = o.a[a] + L - 1; }
                else { lo[a] = o.a[a] - r; hi[a] = o.a[a] + r - 1; }
            }
            int u = ax == 0 ? 1 : 0, v = ax == 2 ? 1 : 2;
            for (int k = lo[2]; k <= hi[2]; k++)
                for (int j = lo[1]; j <= hi[1]; j++)
                    for (int i = lo[0]; i <= hi[0]; i++) {
                        const int idx[3] = {i, j, k};
                        float p = (float)idx[u] - (float)o.a[u] + 0.5f, q = (float)idx[v] - (float)o.a[v] + 0.5f;
                        if ((p * p + q * q) <= (float)r * (float)r) put(i, j, k);
                    }
        }
    }

    // sheets, ref :2290-2352 (sheet materials carry ep = 1 and one sigma)
    SheetCells sc;
    int smid = 0;
    for (auto& s : d.sheets) {
        for (size_t r = 0; r < d.smats.size(); r++) if ((float)s.mat == d.smats[r].id) smid = (int)r + 1;
        if (smid == 0) continue;
        const float sg = d.smats[smid - 1].sig[0];
        int ua = s.normal == 0 ? 1 : 0, ub = s.normal == 2 ? 1 : 2;
        auto& pl = sc.plane[s.normal][s.pos];
        if (pl.empty()) pl.assign((size_t)m.S[ua] * m.S[ub], 0.0f);
        for (int b = s.start[1]; b <= s.start[1] + s.len[1] - 1; b++)
            for (int a = s.start[0]; a <= s.start[0] + s.len[0] - 1; a++) {
                int idx[3];
                idx[s.normal] = s.pos; idx[ua] = a; idx[ub] = b;
                if (cell_ok(idx[0], idx[1], idx[2])) pl[(size_t)m.pos(ub, b) * m.S[ua] + m.pos(ua, a)] = sg;
                if (float* g = geo(1 + s.normal, idx[0], idx[1], idx[2])) *g = (float)s.mat;
            }
    }
    // sheet cell sigma with the PBC mapping; non-sheet cells are 0
    auto sheet_sig_cell = [&](int n, int i, int j, int k) -> float {
        const int idx[3] = {i, j, k};
        int pn = idx[n];
        if (d.pbc[n]) pn = m.pos(n, pn) + 1;
        auto it = sc.plane[n].find(pn);
        if (it == sc.plane[n].end()) return 0.0f;
        int ua = n == 0 ? 1 : 0, ub = n == 2 ? 1 : 2;
        return it->second[(size_t)m.pos(ub, idx[ub]) * m.S[ua] + m.pos(ua, idx[ua])];
    };
    // averaged sheet values of component c for normal n at an edge
    auto sheet_edge = [&](int n, int c, int i, int j, int k, float* ep, float* sg) {
        if (edge_unaveraged(m, i, j, k)) { *ep = 1.0f; *sg = 0.0f; return; }
        int cell[4][3];
        sheet_stencil(n, c, i, j, k, cell);
        float s[4];
        for (int q = 0; q < 4; q++) s[q] = sheet_sig_cell(n, cell[q][0], cell[q][1], cell[q][2]);
        *ep = (1.0f + 1.0f + 1.0f + 1.0f) / 4.0f;
        *sg = (s[0] + s[1] + s[2] + s[3]) / 4.0f;
    };

    // uniform-neighbourhood coefficient table (reference 4-term averages)
    const float dt = d.del_t;
    m.ucoef.assign(m.mats.size(), AemUniformCoef{});
    for (size_t r = 0; r < m.mats.size(); r++) {
        const AemMaterial& am = m.mats[r];
        AemUniformCoef& u = m.ucoef[r];
        for (int c = 0; c < 3; c++) {
            float e = (am.eps[c] + am.eps[c] + am.eps[c] + am.eps[c]) / 4.0f;
            float s = (am.sig[c] + am.sig[c] + am.sig[c] + am.sig[c]) / 4.0f;
            float tp = 0.0f;
            for (int p = 0; p < m.npoles; p++) {
                float w = (am.wp[p][c] + am.wp[p][c] + am.wp[p][c] + am.wp[p][c]) / 4.0f;
                float g = (am.gam[p][c] + am.gam[p][c] + am.gam[p][c] + am.gam[p][c]) / 4.0f;
                u.ja[p][c] = ja_of(g, dt);
                u.jb[p][c] = jb_of(w, g, dt);
            }
            for (int p = 0; p < m.npoles; p++) tp = tp + u.jb[p][c];
            u.ga[c] = ga_of(s + tp, e, dt);
            u.gb[c] = gb_of(s + tp, e, dt);
        }
    }
    // vacuum defaults must match for the unaveraged edges
    m.has_drude = false;

    // sheet planes
    for (int n = 0; n < 3; n++)
        for (auto& kv : sc.plane[n]) {
            SheetPlaneHost sp;
            sp.axis = n; sp.pos = kv.first;
            int ua = n == 0 ? 1 : 0, ub = n == 2 ? 1 : 2;
            sp.na = m.S[ua]; sp.nb = m.S[ub]; sp.pa = sp.na;
            size_t nn = (size_t)sp.na * sp.nb;
            sp.nmask.assign(nn, 0); sp.tmask.assign(nn, 0);
            sp.sa.assign(nn, 0); sp.sb.assign(nn, 0);
            sp.ga1.assign(nn, 0); sp.gb1.assign(nn, 0); sp.ga2.assign(nn, 0); sp.gb2.assign(nn, 0);
            const float dl[3] = {d.dx, d.dy, d.dz};
            for (int pb = 0; pb < sp.nb; pb++)
                for (int pa = 0; pa < sp.na; pa++) {
                    int idx[3];
                    idx[n] = sp.pos; idx[ua] = pa + 1; idx[ub] = pb + 1;
                    size_t q = (size_t)pb * sp.pa + pa;
                    // normal component: E_special coefficients, ref :5722-5726
                    float ep, sg;
                    sheet_edge(n, n, idx[0], idx[1], idx[2], &ep, &sg);
                    if (sg > 0 || ep > 1) {
                        sp.nmask[q] = 1;
                        sp.sa[q] = (1.0f - sg * dt / (2.0f * kEp0 * ep)) / (1.0f + sg * dt / (2.0f * kEp0 * ep));
                        sp.sb[q] = (dt / (kEp0 * ep)) / (1.0f + sg * dt / (2.0f * kEp0 * ep));
                    }
                    // tangential components: thickness-weighted overrides, ref :2930-3005 / :3019-3115
                    const int tc[2] = {ua, ub};
                    for (int t = 0; t < 2; t++) {
                        int c = tc[t];
                        float be_eps, be_sig, wp[AEM_MAX_POLES], gm[AEM_MAX_POLES];
                        edge_material(m, c, idx[0], idx[1], idx[2], &be_eps, &be_sig, wp, gm);
                        float ea = be_eps, sa = be_sig;
                        int hit = 0;
                        for (int n2 = 0; n2 < 3; n2++) {
                            if (n2 == c || sc.plane[n2].empty()) continue;
                            float se, ss;
                            sheet_edge(n2, c, idx[0], idx[1], idx[2], &se, &ss);
                            if (ss > 0 || se > 1) {
                                ea = ea + (d.sheet_thickness / dl[n2]) * (se - be_eps);
                                sa = sa + (d.sheet_thickness / dl[n2]) * (ss - be_sig);
                                hit = 1;
                            }
                        }
                        if (!hit) continue;
                        float tp = 0.0f;
                        for (int p = 0; p < m.npoles; p++) tp = tp + jb_of(wp[p], gm[p], dt);
                        sp.tmask[q] |= (uint8_t)(1 << t);
                        float g_a = ga_of(sa + tp, ea, dt), g_b = gb_of(sa + tp, ea, dt);
                        if (t == 0) { sp.ga1[q] = g_a; sp.gb1[q] = g_b; }
                        else { sp.ga2[q] = g_a; sp.gb2[q] = g_b; }
                    }
                }
            m.splanes.push_back(std::move(sp));
        }
    if (m.splanes.size() > AEM_MAX_SHEET_PLANES) throw DeckError("too many distinct sheet planes");

    // Drude bounding boxes, ref :3126-3248
    if (is_plasma) {
        bool any = false;
        for (int c = 0; c < 3; c++) {
            int* bx = m.dbox[c];
            bx[0] = N[2] - 1; bx[1] = c == 2 ? 1 : 2;
            bx[2] = N[1] - 1; bx[3] = c == 1 ? 1 : 2;
            bx[4] = N[0] - 1; bx[5] = c == 0 ? 1 : 2;
            int k0 = c == 2 ? 1 : 2, j0 = c == 1 ? 1 : 2, i0 = c == 0 ? 1 : 2;
            float eps, sig, wp[AEM_MAX_POLES], gm[AEM_MAX_POLES];
            for (int k = k0; k <= N[2] - 1; k++)
                for (int j = j0; j <= N[1] - 1; j++)
                    for (int i = i0; i <= N[0] - 1; i++) {
                        edge_material(m, c, i, j, k, &eps, &sig, wp, gm);
                        bool hit = false;
                        for (int p = 0; p < m.npoles && !hit; p++)
                            if (ja_of(gm[p], dt) > 1 || jb_of(wp[p], gm[p], dt) > 0) hit = true;
                        if (!hit) continue;
                        any = true;
                        bx[0] = std::min(bx[0], k); bx[1] = std::max(bx[1], k);
                        bx[2] = std::min(bx[2], j); bx[3] = std::max(bx[3], j);
                        bx[4] = std::min(bx[4], i); bx[5] = std::max(bx[5], i);
                    }
        }
        m.has_drude = any && m.npoles > 0;
    }

    // CPML tables, ref :3404-3577, den_*, ref :3586-3666
    const float dl[3] = {d.dx, d.dy, d.dz};
    float kap_e[3][2][AEM_MAX_PML + 1] = {}, kap_h[3][2][AEM_MAX_PML + 1] = {};
    // g^m as the reference writes it for m = 3, ((g*g)*g); other orders
    // (extension cpml_grading) multiply on in the same left-to-right order
    auto gpow = [&](float g) {
        float p = g;
        for (int q = 1; q < d.cpml_m; q++) p = p * g;
        return p;
    };
    for (int a = 0; a < 3; a++)
        for (int s = 0; s < 2; s++) {
            int n = d.npml[a][s];
            if (n > AEM_MAX_PML) throw DeckError("CPML too thick");
            for (int i = 1; i <= n; i++) {
                float g = (float)(n - i) / ((float)n - 1.0f);
                float sg = d.sig_max[a] * gpow(g);
                float al = d.alpha_max * (((float)i - 1.0f) / ((float)n - 1.0f));
                float ka = 1.0f + (d.kappa_max - 1.0f) * gpow(g);
                float b = std::exp(-((sg / ka + al) * dt / kEp0));
                float c = (sg == 0.0f && al == 0.0f && i == n) ? 0.0f : sg * (b - 1.0f) / (sg + ka * al) / ka;
                m.be[a][s][i - 1] = b; m.ce[a][s][i - 1] = c; kap_e[a][s][i] = ka;
            }
            for (int i = 1; i <= n - 1; i++) {
                float g = ((float)(n - i) - 0.5f) / ((float)n - 1.0f);
                float sg = d.sig_max[a] * gpow(g);
                float al = d.alpha_max * (((float)i - 0.5f) / ((float)n - 1.0f));
                float ka = 1.0f + (d.kappa_max - 1.0f) * gpow(g);
                float b = std::exp(-((sg / ka + al) * dt / kEp0));
                float c = sg * (b - 1.0f) / (sg + ka * al) / ka;
                m.bh[a][s][i - 1] = b; m.ch[a][s][i - 1] = c; kap_h[a][s][i] = ka;
            }
            (void)s;
        }
    for (int a = 0; a < 3; a++) {
        int n1 = d.npml[a][0], n2 = d.npml[a][1];
        m.den_h[a].assign((size_t)N[a] + 1, 0.0f);
        m.den_e[a].assign((size_t)N[a] + 1, 0.0f);
        int q = n2 - 1;
        for (int i = 1; i <= N[a] - 1; i++) {
            float v;
            if (i <= n1 - 1) v = 1.0f / (kap_h[a][0][i] * dl[a]);
            else if (i >= N[a] + 1 - n2) { v = 1.0f / (kap_h[a][1][q] * dl[a]); q--; }
            else v = 1.0f / dl[a];
            m.den_h[a][i - 1] = v;
        }
        q = n2;
        for (int i = 1; i <= N[a] - 1; i++) {
            float v;
            if (i <= n1) v = 1.0f / (kap_e[a][0][i] * dl[a]);
            else if (i >= N[a] + 1 - n2) { v = 1.0f / (kap_e[a][1][q] * dl[a]); q--; }
            else v = 1.0f / dl[a];
            m.den_e[a][i - 1] = v;
        }
    }

    // gridded feeds, ref :3723-3744
    m.feeds.assign(d.ports.size(), {});
    int M1 = 0, M2 = 0;
    bool any_grid = false;
    for (auto& p : d.ports) {
        M1 = std::max(M1, (int)p.size[0]);
        M2 = std::max(M2, (int)p.size[1]);
        any_grid |= p.gridded != 0;
    }
    m.feed_m1 = M1 + 1; m.feed_m2 = M2 + 1;
    for (size_t q = 0; q < d.ports.size(); q++) {
        const Port& p = d.ports[q];
        if (!p.gridded) continue;
        int n1 = (int)p.size[0], n2 = (int)p.size[1];
        std::string path = resolve(workdir, p.feed);
        std::ifstream f(path, std::ios::binary);
        if (!f) throw DeckError("cannot open gridded feed file '" + path + "'");
        m.feeds[q].assign((size_t)4 * (n1 + 1) * (n2 + 1), 0.0f);
        f.read((char*)m.feeds[q].data(), (std::streamsize)(m.feeds[q].size() * sizeof(float)));
        if ((size_t)f.gcount() != m.feeds[q].size() * sizeof(float)) throw DeckError("gridded feed file '" + path + "' is too short");
    }
    (void)any_grid;
    if (d.ext_coef64) coef_tables_fp64(m);
}

}  // namespace aem
