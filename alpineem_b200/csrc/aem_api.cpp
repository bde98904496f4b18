// aem_api.cpp -- C ABI over aem::Solver (declared in include/alpineem_b200.h).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

#include "../../include/alpineem_b200.h"
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
    } catch (const std::runtime_error& e) {
        std::string m = e.what();
        return fail(h, m.rfind("CUDA", 0) == 0 ? AEM_ERR_CUDA : AEM_ERR_INPUT, m);
    } catch (const std::exception& e) {
        return fail(h, AEM_ERR_INPUT, e.what());
    }
}
}  // namespace

extern "C" {

int aem_version(void) { return 1 * 10000 + 0 * 100 + 0; }

int aem_create_from_file(const char* inputs_path, int mode, const char* outdir, aem_handle** out) {
    if (!inputs_path || !out || (mode != AEM_STANDARD && mode != AEM_KMAX)) return fail(nullptr, AEM_ERR_ARG, "bad argument");
    *out = nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(nullptr, AEM_ERR_CUDA, "CUDA error: no usable CUDA device");
    return guarded(nullptr, [&]() {
        auto h = std::make_unique<aem_handle>();
        std::string od = outdir ? outdir : "";
        h->s = std::make_unique<aem::Solver>(inputs_path, mode == AEM_KMAX, od);
        // <name>_geometry.bin, ref :2355-2357
        const aem::Deck& d = h->s->deck();
        std::string base = d.filename.substr(0, d.filename.size() >= 4 ? d.filename.size() - 4 : 0);
        std::string fn = (od.empty() ? "" : od + "/") + base + "_geometry.bin";
        if (FILE* f = std::fopen(fn.c_str(), "wb")) {
            const std::vector<float>& g = h->s->geometry();
            std::fwrite(g.data(), sizeof(float), g.size(), f);
            std::fclose(f);
        }
        *out = h.release();
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
    if (!h || !dims || comp < 0 || comp > 5) return fail(h, AEM_ERR_ARG, "bad argument");
    return guarded(h, [&]() {
        std::vector<double> r, i;
        h->s->get_field(comp, r, i, dims);
        if (re) std::memcpy(re, r.data(), sizeof(double) * r.size());
        if (im) std::memcpy(im, i.data(), sizeof(double) * i.size());
        return AEM_OK;
    });
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
