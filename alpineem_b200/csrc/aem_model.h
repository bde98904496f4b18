// aem_model.h -- host-side model built from a Deck: the data that is
// uploaded once to the GPU before the time loop.
#pragma once
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <memory>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "aem_deck.h"
#include "aem_types.h"

namespace aem {

// f(0..n-1) on the host's cores (items handed out one at a time); for
// loops whose iterations write disjoint data
template <typename F>
inline void par_for(int n, F&& f) {
    const unsigned hc = std::thread::hardware_concurrency();
    const int nt = (int)std::min<unsigned>(hc ? hc : 1, 64);
    if (n < 16 || nt <= 1) {
        for (int i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < std::min(nt, n); t++)
        th.emplace_back([&] {
            for (int i; (i = next.fetch_add(1)) < n;) f(i);
        });
    for (auto& x : th) x.join();
}

struct SheetPlaneHost {
    int axis = 0, pos = 0;        // normal axis, reference index along it
    int na = 0, nb = 0, pa = 0;   // in-plane storage extents and pitch
    std::vector<uint8_t> nmask, tmask;
    std::vector<float> sa, sb, ga1, gb1, ga2, gb2;
};

// std::allocator that leaves new elements uninitialised (resize() of a
// multi-GB array need not write it; the model builder fills it in parallel)
template <typename T>
struct DefaultInit : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = DefaultInit<U>;
    };
    template <typename U>
    void construct(U* p) noexcept {
        ::new ((void*)p) U;
    }
    template <typename U, typename... A>
    void construct(U* p, A&&... a) {
        ::new ((void*)p) U(std::forward<A>(a)...);
    }
};

struct HostModel {
    Deck d;
    int S[3] = {0, 0, 0};   // storage extents per axis
    int PX = 0;             // x pitch
    long long plane = 0, cells = 0;
    std::vector<uint8_t, DefaultInit<uint8_t>> cell_id;  // [SZ][SY][PX], 0 = vacuum
    std::vector<AemMaterial> mats;                // 0 = vacuum, 1.. = deck volume materials
    std::vector<AemUniformCoef> ucoef;            // same indexing
    int npoles = 0;
    bool has_drude = false;
    int dbox[3][6] = {};                          // Drude boxes (reference indices)
    std::vector<SheetPlaneHost> splanes;
    std::vector<float> den_e[3], den_h[3];        // index 0..N-1 holds den(1..N-1) at [idx-1]
    float be[3][2][AEM_MAX_PML] = {}, ce[3][2][AEM_MAX_PML] = {};
    float bh[3][2][AEM_MAX_PML] = {}, ch[3][2][AEM_MAX_PML] = {};
    std::vector<std::vector<float>> feeds;        // per port: gridded feed (4, n1+1, n2+1), F-order
    int feed_m1 = 0, feed_m2 = 0;                 // reference array extents (max n1+1, max n2+1)
    std::vector<float> geometry;                  // (4, gx, gy, gz) F-order float32 for _geometry.bin
    // When no host step reads the ids (no sheets, no Drude poles, no
    // _geometry.bin) cell_id stays empty and the ids are rasterised on the
    // device (rasterise_device): raster_bulk points at the bulk ids in the
    // file's layout (the caller's buffer or raster_file) and raster_map
    // maps a file id to its material index.  Valid until the solver's setup
    // has uploaded them.
    bool raster_device = false;
    const float* raster_bulk = nullptr;
    std::vector<float> raster_file;
    std::vector<int> raster_map;

    // storage position of reference index `idx` on axis a (wraps when periodic)
    int pos(int a, int idx) const {
        if (d.pbc[a]) {
            int n = S[a];
            int p = (idx - 1) % n;
            return p < 0 ? p + n : p;
        }
        return idx - 1;
    }
    long long lin(int i, int j, int k) const {  // reference cell/edge indices
        return ((long long)pos(2, k) * S[1] + pos(1, j)) * PX + pos(0, i);
    }
};

// Build the model: geometry rasterisation, material tables, sheets, Drude
// boxes, CPML tables and gridded feeds.  `workdir` resolves relative file
// names (bulk geometry, gridded feeds).  Throws DeckError.
// `bulk`, when not null, replaces the deck's bulk geometry file: `bulk_n`
// float32 material ids in the file's layout (x fastest).
void build_model(HostModel& m, const std::string& workdir, const float* bulk = nullptr, size_t bulk_n = 0);

// Extension `coef_precision 64`: recompute the material (Ga, Gb, Drude Ja,
// Jb), CPML (b, c) and den tables on the current CUDA device in FP64, each
// rounded to FP32 once (aem_coef.cu).  Throws std::runtime_error on a CUDA
// failure.
void coef_tables_fp64(HostModel& m);

// The per-cell material ids of a model built with raster_device set,
// written into the zeroed device array `cell` ([SZ][SY][PX]) on stream `s`
// (aem_raster.cu): the same ids the host builder writes.  Adds the bytes
// copied to the device to `h2d`; returns after the stream has finished.
// Throws std::runtime_error on a CUDA failure.
void rasterise_device(const HostModel& m, uint8_t* cell, struct CUstream_st* s, size_t& h2d);

// Edge coefficients as the reference computes them from the averaged cell
// properties (used by the host for sheet overrides and by tests).
void edge_material(const HostModel& m, int comp, int i, int j, int k, float* eps, float* sig,
                   float* wp /*[npoles]*/, float* gam /*[npoles]*/);

}  // namespace aem
