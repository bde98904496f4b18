// aem_api.cpp -- C ABI over aem::Solver (declared in include/alpineem_b200.h).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>
#include <stdexcept>
#include <string>

#include "../../include/alpineem_b200.h"
#include "aem_design.h"
#include "aem_dft.h"
#include "aem_solver.h"

struct aem_handle {
    std::unique_ptr<aem::Solver> s;
    std::string err;
    bool written = false;
};

namespace {
thread_local std::string g_create_err;

int fail(aem_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    else g_create_err = msg;
    return code;
}

template <typename F>
int guarded(aem_handle* h, F&& f) {
    try {
        return f();
    } catch (const aem::DeckError& e) {
        return fail(h, AEM_ERR_INPUT, e.what());
    } catch (const aem::Diverged& e) {
        return fail(h, AEM_ERR_DIVERGED, e.what());
    } catch (const std::invalid_argument& e) {
        return fail(h, AEM_ERR_ARG, e.what());
    } catch (const std::runtime_error& e) {
        std::string m = e.what();
        return fail(h, m.rfind("CUDA", 0) == 0 ? AEM_ERR_CUDA : AEM_ERR_INPUT, m);
    } catch (const std::exception& e) {
        return fail(h, AEM_ERR_INPUT, e.what());
    }
}
}  // namespace

namespace aem {
// error text for entry points that have no handle (aem_last_error(NULL))
void set_global_error(const std::string& msg) { g_create_err = msg; }
}  // namespace aem

extern "C" {

int aem_version(void) { return 1 * 10000 + 0 * 100 + 0; }

// <name>_geometry.bin, ref :2355-2357 (skipped with the geometry_bin no extension)
static void write_geometry(const aem::Solver& s, const std::string& od) {
    const aem::Deck& d = s.deck();
    if (!d.ext_geometry_bin) return;
    std::string base = d.filename.substr(0, d.filename.size() >= 4 ? d.filename.size() - 4 : 0);
    std::string fn = (od.empty() ? "" : od + "/") + base + "_geometry.bin";
    FILE* f = std::fopen(fn.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write '" + fn + "'");
    const std::vector<float>& g = s.geometry();
    size_t w = std::fwrite(g.data(), sizeof(float), g.size(), f);
    std::fclose(f);
    if (w != g.size()) throw std::runtime_error("short write to '" + fn + "'");
}

static int need_device() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, AEM_ERR_CUDA, "CUDA error: no usable CUDA device");
    }
    return AEM_OK;
}

int aem_create_from_file(const char* inputs_path, int mode, const char* outdir, aem_handle** out) {
    if (!inputs_path || !out || (mode != AEM_STANDARD && mode != AEM_KMAX)) return fail(nullptr, AEM_ERR_ARG, "bad argument");
    *out = nullptr;
    if (int rc = need_device()) return rc;
    return guarded(nullptr, [&]() {
        auto h = std::make_unique<aem_handle>();
        std::string od = outdir ? outdir : "";
        h->s = std::make_unique<aem::Solver>(inputs_path, mode == AEM_KMAX, od);
        write_geometry(*h->s, od);
        *out = h.release();
        return AEM_OK;
    });
}

int aem_create_from_memory(const char* deck_text, const char* ext_text, const float* bulk, size_t bulk_count, int mode,
                           const char* outdir, aem_handle** out) {
    if (!deck_text || !out || (mode != AEM_STANDARD && mode != AEM_KMAX) || (bulk_count && !bulk))
        return fail(nullptr, AEM_ERR_ARG, "bad argument");
    *out = nullptr;
    if (int rc = need_device()) return rc;
    return guarded(nullptr, [&]() {
        auto h = std::make_unique<aem_handle>();
        std::string od = outdir ? outdir : "";
        h->s = std::make_unique<aem::Solver>(deck_text, ext_text ? ext_text : "", bulk, bulk_count, mode == AEM_KMAX, od, od);
        write_geometry(*h->s, od);
        *out = h.release();
        return AEM_OK;
    });
}

int aem_check_deck(const char* deck_text, const char* ext_text, int mode, int sizes[3]) {
    if (!deck_text || (mode != AEM_STANDARD && mode != AEM_KMAX)) return fail(nullptr, AEM_ERR_ARG, "bad argument");
    return guarded(nullptr, [&]() {
        aem::Deck d = aem::parse_deck(deck_text, mode == AEM_KMAX);
        aem::apply_extensions(d, ext_text ? ext_text : "");
        aem::derive(d);
        if (sizes) { sizes[0] = d.X; sizes[1] = d.Y; sizes[2] = d.Z; }
        return AEM_OK;
    });
}

int aem_run(aem_handle* h, int nsteps) {
    if (!h || nsteps < 0) return fail(h, AEM_ERR_ARG, "bad argument");
    return guarded(h, [&]() {
        h->s->run(nsteps);
        return AEM_OK;
    });
}

int aem_autotune(aem_handle* h, int steps_per_candidate, int shape[4]) {
    if (!h || steps_per_candidate < 0) return fail(h, AEM_ERR_ARG, "bad argument");
    return guarded(h, [&]() {
        h->s->autotune(steps_per_candidate, shape);
        return AEM_OK;
    });
}

int aem_run_graph(aem_handle* h, int nsteps, int steps_per_graph) {
    if (!h || nsteps < 0 || steps_per_graph < 1) return fail(h, AEM_ERR_ARG, "bad argument");
    return guarded(h, [&]() {
        h->s->run_graph(nsteps, steps_per_graph);
        return AEM_OK;
    });
}

int aem_run_batch(aem_handle* const* hs, int count, int nsteps, int steps_per_graph) {
    if (!hs || count < 1 || nsteps < 0 || steps_per_graph < 1) return fail(nullptr, AEM_ERR_ARG, "bad argument");
    std::vector<aem::Solver*> v(count);
    for (int i = 0; i < count; i++) {
        if (!hs[i]) return fail(nullptr, AEM_ERR_ARG, "bad argument");
        v[i] = hs[i]->s.get();
    }
    return guarded(nullptr, [&]() {
        aem::Solver::run_batch(v.data(), count, nsteps, steps_per_graph);
        return AEM_OK;
    });
}

int aem_steps(aem_handle* h, int* done, int* total) {
    if (!h) return AEM_ERR_ARG;
    if (done) *done = h->s->steps_done();
    if (total) *total = h->s->deck().steps;
    return AEM_OK;
}

int aem_synchronize(aem_handle* h) {
    if (!h) return AEM_ERR_ARG;
    cudaError_t e = cudaStreamSynchronize(h->s->stream());
    if (e != cudaSuccess) return fail(h, AEM_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    return AEM_OK;
}

int aem_write_outputs(aem_handle* h) {
    if (!h) return AEM_ERR_ARG;
    if (h->s->steps_done() != h->s->deck().steps) return fail(h, AEM_ERR_STATE, "outputs need every time step to be run first");
    return guarded(h, [&]() {
        h->s->finalize_and_write();
        h->written = true;
        return AEM_OK;
    });
}

int aem_get_series(aem_handle* h, int kind, int index, double* re, double* im, int n) {
    if (!h || !re || n < 0) return fail(h, AEM_ERR_ARG, "bad argument");
    if (!h->written) return fail(h, AEM_ERR_STATE, "series are available after aem_write_outputs");
    aem::Solver& s = *h->s;
    const std::vector<double>* r = nullptr;
    const std::vector<double>* i = nullptr;
    switch (kind) {
    case 0: r = &s.incident_re; i = &s.incident_im; break;
    case 1: r = &s.refl_re; i = &s.refl_im; break;
    case 2: r = &s.trans_re; i = &s.trans_im; break;
    case 3: r = &s.refl_tm_re; i = &s.refl_tm_im; break;
    case 4: r = &s.trans_tm_re; i = &s.trans_tm_im; break;
    case 5:
        if (index < 0 || index >= (int)s.vout_re.size()) return fail(h, AEM_ERR_ARG, "no such port");
        r = &s.vout_re[index]; i = &s.vout_im[index]; break;
    case 6:
    case 7:
        if (index < 0 || index >= (int)s.eth_re.size()) return fail(h, AEM_ERR_ARG, "no such far-field angle");
        r = kind == 6 ? &s.eth_re[index] : &s.eph_re[index];
        i = kind == 6 ? &s.eth_im[index] : &s.eph_im[index];
        break;
    default: return fail(h, AEM_ERR_ARG, "unknown series kind");
    }
    int m = (int)r->size() < n ? (int)r->size() : n;
    std::memcpy(re, r->data(), sizeof(double) * m);
    if (im) std::memcpy(im, i->data(), sizeof(double) * m);
    return m;
}

int aem_get_field(aem_handle* h, int comp, int dims[3], double* re, double* im) {
    if (!h || !dims || comp < 0 || comp > 6) return fail(h, AEM_ERR_ARG, "bad argument");
    return guarded(h, [&]() {
        std::vector<double> r, i;
        h->s->get_field(comp, r, i, dims);
        if (re) std::memcpy(re, r.data(), sizeof(double) * r.size());
        if (im) std::memcpy(im, i.data(), sizeof(double) * i.size());
        return AEM_OK;
    });
}

int aem_profile(aem_handle* h, int enable) {
    if (!h) return AEM_ERR_ARG;
    return guarded(h, [&]() {
        h->s->set_profiling(enable != 0);
        return AEM_OK;
    });
}

int aem_profile_read(aem_handle* h, double ms[AEM_NPHASE], long long launches[AEM_NPHASE]) {
    if (!h || !ms || !launches) return fail(h, AEM_ERR_ARG, "bad argument");
    return guarded(h, [&]() {
        h->s->read_profile(ms, launches);
        return AEM_OK;
    });
}

int aem_flush(aem_handle* h) {
    if (!h) return AEM_ERR_ARG;
    return guarded(h, [&]() {
        h->s->flush();
        return AEM_OK;
    });
}

int aem_stream(aem_handle* h, void** stream) {
    if (!h || !stream) return fail(h, AEM_ERR_ARG, "bad argument");
    *stream = (void*)h->s->stream();
    return AEM_OK;
}

int aem_transfer_bytes(aem_handle* h, long long* h2d, long long* d2h) {
    if (!h) return AEM_ERR_ARG;
    if (h2d) *h2d = (long long)h->s->h2d_bytes();
    if (d2h) *d2h = (long long)h->s->d2h_bytes();
    return AEM_OK;
}

int aem_launch_count(aem_handle* h, long long* n) {
    if (!h || !n) return fail(h, AEM_ERR_ARG, "bad argument");
    *n = h->s->launches();
    return AEM_OK;
}

int aem_read_probe(aem_handle* h, int kind, int index, int first_step, int n, double* re, double* im) {
    if (!h || !re || n < 0) return fail(h, AEM_ERR_ARG, "bad argument");
    return guarded(h, [&]() {
        h->s->read_probe(kind, index, first_step, n, re, im);
        return AEM_OK;
    });
}

int aem_read_spectrum(aem_handle* h, int kind, int index, int n, double* freqs, double* re, double* im) {
    if (!h || !re || n < 0) return fail(h, AEM_ERR_ARG, "bad argument");
    return guarded(h, [&]() { return h->s->read_spectrum(kind, index, n, freqs, re, im); });
}

int aem_checkpoint_save(aem_handle* h, const char* path) {
    if (!h || !path) return fail(h, AEM_ERR_ARG, "bad argument");
    return guarded(h, [&]() {
        h->s->checkpoint_save(path);
        return AEM_OK;
    });
}

int aem_checkpoint_load(aem_handle* h, const char* path) {
    if (!h || !path) return fail(h, AEM_ERR_ARG, "bad argument");
    return guarded(h, [&]() {
        h->s->checkpoint_load(path);
        return AEM_OK;
    });
}

int aem_time_step(aem_handle* h, double* dt) {
    if (!h || !dt) return fail(h, AEM_ERR_ARG, "bad argument");
    *dt = (double)h->s->model().d.del_t;
    return AEM_OK;
}

int aem_workload(aem_handle* h, long long* cells, double* bytes_per_step) {
    if (!h) return AEM_ERR_ARG;
    if (cells) *cells = h->s->cell_count();
    if (bytes_per_step) *bytes_per_step = h->s->algorithmic_bytes_per_step();
    return AEM_OK;
}

int aem_far_field_size(aem_handle* h, long long* face_cells, int* angles) {
    if (!h) return AEM_ERR_ARG;
    long long fc = 0;
    int na = 0;
    h->s->far_field_size(&fc, &na);
    if (face_cells) *face_cells = fc;
    if (angles) *angles = na;
    return AEM_OK;
}

int aem_dft(const float* x, long long n, double dt, const double* freqs, int nf, double* out, void* stream) {
    if (!x || !freqs || !out || n < 1 || nf < 1 || !(dt > 0.0)) return fail(nullptr, AEM_ERR_ARG, "bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    const int chunks = aem::dft_chunks(n, nf);
    double* scratch = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&scratch, sizeof(double) * 2 * (size_t)chunks * nf, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, AEM_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    }
    e = aem::dft_launch(x, n, dt, freqs, nf, out, scratch, chunks, s);
    cudaError_t e2 = cudaFreeAsync(scratch, s);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, AEM_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    }
    return AEM_OK;
}

int aem_dft_batch(const double* x, long long ld, int nseries, long long n, double dt, const double* freqs, int nf,
                  double* out, void* stream) {
    if (!x || !freqs || !out || n < 1 || nf < 1 || nseries < 1 || ld < n || !(dt > 0.0))
        return fail(nullptr, AEM_ERR_ARG, "bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    const int chunks = aem::dftb_chunks(n, nseries, nf);
    double* scratch = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&scratch, sizeof(double) * 2 * (size_t)chunks * nseries * nf, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, AEM_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    }
    e = aem::dftb_launch(x, ld, nseries, n, dt, freqs, nf, out, scratch, chunks, s);
    cudaError_t e2 = cudaFreeAsync(scratch, s);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, AEM_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
    }
    return AEM_OK;
}

int aem_grid(aem_handle* h, int sizes[3]) {
    if (!h || !sizes) return AEM_ERR_ARG;
    const aem::Deck& d = h->s->deck();
    sizes[0] = d.X; sizes[1] = d.Y; sizes[2] = d.Z;
    return AEM_OK;
}

int aem_device_bytes(aem_handle* h, size_t* bytes) {
    if (!h || !bytes) return AEM_ERR_ARG;
    *bytes = h->s->device_bytes();
    return AEM_OK;
}

const char* aem_last_error(aem_handle* h) { return h ? h->err.c_str() : g_create_err.c_str(); }

int aem_destroy(aem_handle* h) {
    delete h;
    return AEM_OK;
}

}  // extern "C"

struct aem_design {
    std::unique_ptr<aem::DesignRun> r;
    std::string err;
};

namespace {
template <typename F>
int dguard(aem_design* d, F&& f) {
    try {
        return f();
    } catch (const aem::DeckError& e) {
        (d ? d->err : g_create_err) = e.what();
        return AEM_ERR_INPUT;
    } catch (const std::invalid_argument& e) {
        (d ? d->err : g_create_err) = e.what();
        return AEM_ERR_ARG;
    } catch (const std::exception& e) {
        std::string m = e.what();
        (d ? d->err : g_create_err) = m;
        return m.rfind("CUDA", 0) == 0 ? AEM_ERR_CUDA : AEM_ERR_INPUT;
    }
}
}  // namespace

extern "C" {

int aem_design_create(const char* inputs_path, const char* outdir, const int lo[3], const int n[3], int precision,
                      aem_design** out) {
    if (!inputs_path || !lo || !n || !out) return fail(nullptr, AEM_ERR_ARG, "bad argument");
    *out = nullptr;
    if (int rc = need_device()) return rc;
    return dguard(nullptr, [&]() {
        auto d = std::make_unique<aem_design>();
        d->r.reset(aem::DesignRun::create(inputs_path, outdir ? outdir : "", lo, n, precision));
        *out = d.release();
        return AEM_OK;
    });
}

int aem_design_set_probe(aem_design* d, int comp, int i, int j, int k, double freq_hz) {
    if (!d) return AEM_ERR_ARG;
    return dguard(d, [&]() {
        d->r->set_probe(comp, i, j, k, freq_hz);
        return AEM_OK;
    });
}

int aem_design_set_eps(aem_design* d, const float* eps, const float* sigma) {
    if (!d) return AEM_ERR_ARG;
    return dguard(d, [&]() {
        d->r->set_design(eps, sigma);
        return AEM_OK;
    });
}

int aem_design_forward(aem_design* d, int checkpoint_every, double* fom, double dft[2]) {
    if (!d || !fom) return AEM_ERR_ARG;
    return dguard(d, [&]() {
        *fom = d->r->forward(checkpoint_every, dft);
        return AEM_OK;
    });
}

int aem_design_gradient(aem_design* d, float* grad_eps, float* grad_sigma, double scale) {
    if (!d) return AEM_ERR_ARG;
    return dguard(d, [&]() {
        d->r->gradient(grad_eps, grad_sigma, scale);
        return AEM_OK;
    });
}

int aem_design_set_overlap(aem_design* d, int enable) {
    if (!d) return AEM_ERR_ARG;
    return dguard(d, [&]() {
        d->r->set_overlap(enable != 0);
        return AEM_OK;
    });
}

int aem_design_gradient_overlap(aem_design* d, float* grad_eps, float* grad_sigma, double scale) {
    if (!d) return AEM_ERR_ARG;
    return dguard(d, [&]() {
        d->r->gradient_overlap(grad_eps, grad_sigma, scale);
        return AEM_OK;
    });
}

int aem_design_timing(aem_design* d, double ms[2], long long launches[2]) {
    if (!d || !ms || !launches) return AEM_ERR_ARG;
    d->r->timing(ms, launches);
    return AEM_OK;
}

int aem_design_get_field(aem_design* d, int comp, int dims[3], double* out) {
    if (!d || !dims) return AEM_ERR_ARG;
    return dguard(d, [&]() {
        std::vector<double> v;
        d->r->get_field(comp, v, dims);
        if (out) std::memcpy(out, v.data(), v.size() * sizeof(double));
        return AEM_OK;
    });
}

int aem_design_stream(aem_design* d, void** stream) {
    if (!d || !stream) return AEM_ERR_ARG;
    *stream = d->r->stream();
    return AEM_OK;
}

const char* aem_design_last_error(aem_design* d) { return d ? d->err.c_str() : g_create_err.c_str(); }

int aem_design_destroy(aem_design* d) {
    delete d;
    return AEM_OK;
}

}  // extern "C"
