// aem_solver.h -- one FDTD run on one GPU: the device state of a deck and
// the per-step launch sequence.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "../../include/alpineem_b200.h"  // AEM_PHASE_*
#include "aem_kernels.h"
#include "aem_model.h"

namespace aem {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

class Solver {
   public:
    // Parse `inputs_path` (relative files resolve against its directory),
    // build the model and upload it to the current CUDA device.
    Solver(const std::string& inputs_path, bool kmax, const std::string& outdir);
    // Same from memory: the deck text, extension lines, and the bulk
    // geometry values when the deck names a bulk file (else null).
    Solver(const std::string& deck_text, const std::string& ext_text, const float* bulk, size_t bulk_n, bool kmax,
           const std::string& outdir, const std::string& workdir);
    ~Solver();
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    // advance `n` time steps (bounded by the deck's step count)
    void run(int n);
    // Advance `n` steps, replaying a captured CUDA graph of `g` steps for
    // every whole chunk: the kernels read the step number from a device
    // counter, so one graph serves every chunk.  Steps before the first chunk
    // (the first step of a run; far-field batch alignment) and after the last
    // run eagerly.  Graph chunks need g even on the fused path (the field
    // buffers swap each step) and g a multiple of the far-field batch.
    void run_graph(int n, int g);
    // Launch shape of the two-kernel update, chosen by timing candidate
    // shapes (z planes and rows per CTA) on the run's own next steps, up to
    // `per` steps each; the fields do not depend on the shape.  Returns
    // (z planes H, rows H, z planes E, rows E).  The fused path has nothing
    // to tune.  The extension `autotune N` runs this at the first step.
    void autotune(int per, int out[4], int budget = 1 << 30);
    // the extension's tuning if it has not run yet, within `budget` steps;
    // returns the steps it ran
    int autotune_pending(int budget);
    // whole-run snapshot (device buffers of the setup, step counters) to a
    // file, and its restore into a handle made from the same deck
    void checkpoint_save(const std::string& path);
    void checkpoint_load(const std::string& path);
    // the launch part of run_graph for a batch of solvers on their own
    // streams: every solver gets to the same point, then the chunks of all
    // solvers are launched round-robin so that their graphs overlap
    static void run_batch(Solver* const* s, int count, int n, int g);
    // post-loop processing and the reference output files (.dat, video)
    void finalize_and_write();
    // host copy of a final field component in the reference layout
    // (comp 0..5 = Ex,Ey,Ez,Hx,Hy,Hz; real part and imaginary part (kmax))
    void get_field(int comp, std::vector<double>& re, std::vector<double>& im, int dims[3]);

    const Deck& deck() const { return m_.d; }
    // device constants, ports and host model (read by the design-gradient
    // engine, which runs its own state over the same grid)
    const AemParams& params() const { return P_; }
    const PortSet& ports() const { return PS_; }
    const HostModel& model() const { return m_; }
    bool port_in_cpml() const { return split_; }
    const std::vector<float>& geometry() const { return m_.geometry; }
    int steps_done() const { return done_; }
    size_t device_bytes() const { return dev_bytes_; }
    cudaStream_t stream() const { return stream_; }
    bool fused() const { return fused_; }
    // kernels launched so far
    long long launches() const { return launches_; }
    // bytes copied host->device (model upload) and device->host so far
    size_t h2d_bytes() const { return h2d_bytes_; }
    size_t d2h_bytes() const { return d2h_bytes_; }
    // bin far-field contributions still held in the batch buffer
    void flush() {
        flush_farfield(done_);
        flush_farfield_tail();
    }
    // per-phase device time: with profiling on, every launcher is bracketed
    // by CUDA events on the solver's stream; read_profile sums them
    void set_profiling(bool on);
    void read_profile(double ms[AEM_NPHASE], long long launches[AEM_NPHASE]);
    // raw per-step samples on the device: port voltage (kind 5, Voltage_out)
    // or unnormalised plane sums (kind 1 reflected, 2 transmitted)
    void read_probe(int kind, int index, int first, int n, double* re, double* im);
    int read_spectrum(int kind, int index, int n, double* freqs, double* re, double* im);
    // bytes the fused Yee/CPML update must move per step (algorithmic)
    double algorithmic_bytes_per_step() const;
    // Huygens-surface cells (both planes of each axis) and far-field angles
    void far_field_size(long long* face_cells, int* angles) const {
        *face_cells = 2 * (FF_.face_n[0] + FF_.face_n[1] + FF_.face_n[2]);
        *angles = FF_.nang;
    }
    long long cell_count() const;

    // time series gathered on the host by finalize
    std::vector<double> incident_re, incident_im;
    std::vector<std::vector<double>> vout_re, vout_im;             // per port
    std::vector<double> refl_re, refl_im, trans_re, trans_im;      // plane sums (TE for kmax)
    std::vector<double> refl_tm_re, refl_tm_im, trans_tm_re, trans_tm_im;
    std::vector<std::vector<double>> eth_re, eth_im, eph_re, eph_im;  // far field, per angle
    std::vector<int> data_out_time;
    std::vector<double> pc_re[3], pc_im[3];

   private:
    void init();
    void release();
    void* alloc(size_t bytes);
    template <typename V, typename A>
    void* upload(const std::vector<V, A>& v);
    void setup_params();
    void setup_ports();
    void setup_farfield();
    void setup_taps();
    void setup_fused();
    void setup_full();
    void step(int counter);
    void flush_farfield(int last);
    void flush_farfield_tail();
    void flush_farfield_last(int last);
    void bin_farfield(int n0, int nt, int carry, bool tail);
    bool graph_ready(int g) const;  // can a g-step graph chunk start at the next step?
    void full_tap(int counter);
    void full_drain(int b);
    void full_flush();
    void capture_graph(int g);
    void release_graph();
    void watchdog_check();
    template <typename Fn>
    void phase(int ph, Fn&& fn);
    cudaEvent_t prof_event();

    std::string outdir_;
    HostModel m_;
    AemParams P_{};
    PortSet PS_{};
    FarFieldDev FF_{};
    TapDev TP_{};
    std::vector<void*> bufs_;
    std::vector<size_t> buf_bytes_;  // size of each buffer of bufs_
    size_t nstate_ = 0;              // buffers allocated by init(): the run's device state
    size_t dev_bytes_ = 0;
    int es_ = 4;  // bytes per field value
    int done_ = 0;
    bool fused_ = false;  // one fused H+E kernel per step (k_yee)
    bool tuned_ = false;  // the two-kernel launch shape has been tuned (or need not be)
    bool split_ = false;  // bulk / port / CPML passes (a port inside a CPML slab)
    AemParams split_params_[2];
    int ff_n0_ = 1;  // first step held in the far-field difference buffer
    size_t ff_part_bytes_ = 0;  // far-field window sums of one batch (scratch)
    // far-field angle whose bins angle q copies (q itself unless q is a
    // second angle of the same direction, e.g. a pole at another phi)
    std::vector<int> ff_canon_;
    std::vector<std::pair<int, int>> dft_series_;  // (probe kind, index) of each on-the-fly spectrum
    long long launches_ = 0;
    size_t h2d_bytes_ = 0, d2h_bytes_ = 0;
    struct ProfMark {
        int phase, n;
        cudaEvent_t e0, e1;
    };
    bool prof_on_ = false;
    std::vector<cudaEvent_t> prof_pool_;
    size_t prof_used_ = 0;
    std::vector<ProfMark> prof_marks_;
    cudaStream_t stream_ = nullptr;
    // graph replay
    int* dstep_ = nullptr;          // device step counter
    int* wd_flag_ = nullptr;        // watchdog: set by k_nonfinite
    cudaGraphExec_t graph_ = nullptr;
    // full-field export (every step's averaged fields to <name>_full_*.bin):
    // the averages go to a device staging buffer, a second stream copies
    // them to pinned host memory, and the host writes them to the files two
    // steps later; two buffers of each, so the copy and the file write of
    // one step overlap the kernels of the next
    struct FullExport {
        int n[3] = {0, 0, 0};      // averaged cells along x, y, z
        size_t bytes = 0;          // one step, six components
        void* dev[2] = {nullptr, nullptr};
        void* host[2] = {nullptr, nullptr};
        cudaEvent_t made[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
        int pending[2] = {0, 0};   // step whose copy buffer b holds (0: none)
        std::FILE* f[6] = {};
        cudaStream_t copy = nullptr;
    } full_;
    int graph_g_ = 0;               // steps per graph
    long long graph_launches_ = 0;  // kernels per replay
};

}  // namespace aem
