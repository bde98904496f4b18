// aem_deck.h -- the solver's input deck (the positional inputs.txt that
// AlpineEM's master.py writes) and the quantities derived from it.
//
// Grammar: main_fdtd/fdtd_solver.f90:726-1298 (annotated template
// main_fdtd/master.py:51-296).  Derived quantities: :1305-1812.
#pragma once
#include <stdexcept>
#include <array>
#include <string>
#include <vector>

namespace aem {

struct DeckError : std::runtime_error {
    explicit DeckError(const std::string& m) : std::runtime_error(m) {}
};

// a run stopped by the watchdog: a non-finite field value
struct Diverged : std::runtime_error {
    using std::runtime_error::runtime_error;
};

struct VolumeMaterial {
    float id = 0;
    float eps[3] = {1, 1, 1};
    float sig[3] = {0, 0, 0};
    int npoles = 0;
    float wp[6][3] = {};
    float gam[6][3] = {};
};

struct SheetMaterial {
    float id = 0;
    float ep[3] = {1, 1, 1};
    float sig[3] = {0, 0, 0};
};

struct Object {
    enum Kind { Block, Sphere, Cylinder } kind;
    int mat = 0;        // material id as written in the deck
    int a[3] = {};      // block: start; sphere: centre; cylinder: start
    int b[3] = {};      // block: lengths; sphere: b[0] = radius; cylinder: b[0]=len, b[1]=radius
    int axis = 0;       // cylinder axis 0/1/2
};

struct Sheet {
    int normal;         // 0/1/2
    int mat;            // sheet material id
    int pos;            // index along the normal
    int start[2], len[2];
};

struct Port {
    int gridded = 0;    // 0 basic, 1 gridded
    int dir = 0;        // axis 0/1/2 (ports(i,1,1))
    int side = 0;       // gridded: -x,+x,-y,+y,-z,+z -> 0..5 (ports(i,1,2))
    float L = 0, C = 0; // line inductance/capacitance per unit length (ports(i,2,2/3))
    float loc[3] = {};  // ports(i,3,:)
    float size[3] = {}; // ports(i,4,:) after the +1 adjustment of :1145-1155
    std::string feed;   // gridded feed file
};

struct Deck {
    bool kmax = false;
    // as read
    int nx = 0, ny = 0, nz = 0;
    float dx = 0, dy = 0, dz = 0;
    int steps = 0;
    float factor = 1, f_center = 0;
    int pulse_type = 0;
    int bc[6] = {};
    int pbc[3] = {};
    int is_mirror = 0, mirror_type = 0, mirror_height = 0;
    std::string excitation;       // "plane wave" / "antenna"
    float pw_amp = 0, pw_delay = 0, theta = 0, phi = 0, pol = 0, theta_m = 0, phi_m = 0;
    float ant_amp = 0, ant_delay = 0;
    int exc_port = 0;
    int mode_type = 0, k_direction = 0;   // kmax
    float kc[3] = {0, 0, 0};              // k_count_x/y/z (rad/m)
    int n_ff = 0, ic = 0, jc = 0, kc_ = 0;
    std::vector<float> ff_theta, ff_phi;  // radians, as the reference stores them
    int video_on = 0, slice_dir = 0, slice_loc = 0;
    std::string export_all = "no";
    std::string filename = "data.dat";
    std::vector<VolumeMaterial> mats;
    std::vector<SheetMaterial> smats;
    float sheet_thickness = 0;
    std::string bulk_file;                // empty = none
    std::vector<Object> objects;
    std::vector<Sheet> sheets;
    std::vector<Port> ports;
    int num_spice_ports = 0;

    // derived, ref :1305-1812
    int X = 0, Y = 0, Z = 0;
    float del_t = 0;
    float r_relay = 0;
    int len_ff = 0, port_array_size = 0;
    int npml[3][2] = {{11, 11}, {11, 11}, {11, 11}};
    int vid1 = 0, vid2 = 0;
    int lo[3] = {}, hi[3] = {};
    float wall_lo[3] = {1, 1, 1}, wall_hi[3] = {1, 1, 1};
    float mir_off[3] = {}, use_mir[3] = {};
    float M_mir[3] = {1, 1, 1}, J_mir[3] = {1, 1, 1};
    int delay[3] = {}, delay_m[3] = {};
    float WE[3] = {}, WH[3] = {}, WE_m[3] = {}, WH_m[3] = {};
    int ff_lo[3] = {}, ff_hi[3] = {};
    float sig_max[3] = {}, alpha_max = 0, kappa_max = 7;
    float spread = 0, t_spread = 0, min_steps = 0;
    float f_adj = 0;
    int k_pl_H = 0, k_pl_E = 0;
    float knum[3] = {};

    // extensions (sidecar "<inputs>.b200", or the text passed to
    // aem_create_from_memory), one "key value" per line:
    //   pml_cells N      CPML thickness in cells (0 = reference default, 10)
    //   geometry_bin no  do not build or write <name>_geometry.bin
    int ext_pml_cells = 0;
    bool ext_geometry_bin = true;
    std::vector<double> ext_dft_freqs;  // on-the-fly spectra of the per-step series (Hz)
    int ext_watchdog = 0;               // steps between non-finite field checks (0: off)
    //   cpml_grading m sigma_factor kappa_max alpha_max   CPML profile:
    //       polynomial order m, sigma_max = sigma_factor (m+1) / (eta0 d),
    //       kappa and alpha maxima (absent: the reference's fixed profile)
    //   tfsf_inset N     TF/SF planes at index N and X-N (reference: npml+3)
    //   probe i j k      cell-centred Ex, Ey, Ez at cell (i, j, k) every step
    bool ext_cpml = false;
    int ext_cpml_m = 3;
    float ext_cpml_sigma = 0, ext_cpml_kappa = 1, ext_cpml_alpha = 0;
    int ext_tfsf_inset = 0;
    std::vector<std::array<int, 3>> ext_probes;
    int cpml_m = 3;                     // grading order used by the CPML tables
    int ext_autotune = 0;               // autotune N: steps per candidate launch shape (0: off)
    bool ext_coef64 = false;            // coef_precision 64: coefficient tables in FP64 on the GPU
};

// Parse an inputs.txt.  `kmax` selects the constant-k periodic grammar
// (the reference's use_kmax_version build).  Throws DeckError with the
// reference's "ERROR: ..." text on invalid input.
Deck parse_deck(const std::string& text, bool kmax);
Deck parse_deck_file(const std::string& path, bool kmax);
// apply extension lines ("key value") to a parsed deck; unknown keys are errors
void apply_extensions(Deck& d, const std::string& text);
void derive(Deck& d);

}  // namespace aem
