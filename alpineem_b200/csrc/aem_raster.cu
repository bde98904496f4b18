// aem_raster.cu -- the per-cell material ids rasterised on the GPU.
//
// Restates the geometry part of the reference setup
// (main_fdtd/fdtd_solver.f90:2051-2288) for the device id array
// [SZ][SY][PX] (uint8, 0 = vacuum):
//   bulk geometry file :2051-2095  every cell takes the material whose id the
//                                  file holds (ids of no volume material: 0)
//   blocks, spheres,   :2101-2288  in deck order, later objects overwrite;
//   cylinders                      sphere / cylinder membership tested at the
//                                  cell centre in FP32, as the reference does
// with the write rules of the host builder (aem_model.cpp): cells 1..N-1 of
// every axis, not the duplicated layer of a periodic axis.  The host keeps
// building the ids when it needs them itself (sheets, Drude poles, the
// <name>_geometry.bin output); otherwise the run's ids are made here and
// the host never holds the array.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>

#include "aem_model.h"

namespace aem {

namespace {

struct Grid {
    int N[3], S[3], pbc[3], PX;
};

__device__ inline int g_pos(const Grid& g, int a, int idx) {
    if (g.pbc[a]) {
        const int n = g.S[a];
        int p = (idx - 1) % n;
        return p < 0 ? p + n : p;
    }
    return idx - 1;
}
__device__ inline long long g_lin(const Grid& g, int i, int j, int k) {
    return ((long long)g_pos(g, 2, k) * g.S[1] + g_pos(g, 1, j)) * g.PX + g_pos(g, 0, i);
}
__device__ inline bool g_cell_ok(const Grid& g, int i, int j, int k) {
    const int idx[3] = {i, j, k};
    for (int a = 0; a < 3; a++) {
        if (idx[a] < 1 || idx[a] > g.N[a] - 1) return false;
        if (g.pbc[a] && idx[a] == g.N[a] - 1) return false;
    }
    return true;
}

// bulk planes k0+1 .. k0+nk (reference indices) from the file's layout
// (x fastest, gx x gy x gz cells)
__global__ void k_bulk_ids(Grid g, const float* bulk, int gx, int gy, int k0, int nk, const int* map, int mx,
                           uint8_t* cell) {
    const long long n = (long long)gx * gy * nk;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % gx) + 1, j = (int)((e / gx) % gy) + 1, k = (int)(e / ((long long)gx * gy)) + k0 + 1;
        const int iv = (int)bulk[e];
        const int mid = (iv >= 0 && iv <= mx) ? map[iv] : 0;
        if (mid != 0) cell[g_lin(g, i, j, k)] = (uint8_t)mid;
    }
}

// one object over its index box lo..hi: 0 block, 1 sphere, 2 cylinder
struct ObjDev {
    int kind, mid, lo[3], hi[3], a[3], r, axis;
};

__global__ void k_object_ids(Grid g, ObjDev o, uint8_t* cell) {
    const int nx = o.hi[0] - o.lo[0] + 1, ny = o.hi[1] - o.lo[1] + 1, nz = o.hi[2] - o.lo[2] + 1;
    const long long n = (long long)nx * ny * nz;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = o.lo[0] + (int)(e % nx), j = o.lo[1] + (int)((e / nx) % ny), k = o.lo[2] + (int)(e / ((long long)nx * ny));
        if (!g_cell_ok(g, i, j, k)) continue;
        bool in = true;
        if (o.kind == 1) {
            const float x = (float)i - (float)o.a[0] + 0.5f, y = (float)j - (float)o.a[1] + 0.5f,
                        z = (float)k - (float)o.a[2] + 0.5f;
            in = (x * x + y * y + z * z) <= (float)o.r * (float)o.r;
        } else if (o.kind == 2) {
            const int idx[3] = {i, j, k};
            const int u = o.axis == 0 ? 1 : 0, v = o.axis == 2 ? 1 : 2;
            const float p = (float)idx[u] - (float)o.a[u] + 0.5f, q = (float)idx[v] - (float)o.a[v] + 0.5f;
            in = (p * p + q * q) <= (float)o.r * (float)o.r;
        }
        if (in) cell[g_lin(g, i, j, k)] = (uint8_t)o.mid;
    }
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e) + " (" + what + ")");
    }
}

}  // namespace

void rasterise_device(const HostModel& m, uint8_t* cell, cudaStream_t s, size_t& h2d) {
    const Deck& d = m.d;
    Grid g;
    const int N[3] = {d.X, d.Y, d.Z};
    for (int a = 0; a < 3; a++) {
        g.N[a] = N[a];
        g.S[a] = m.S[a];
        g.pbc[a] = d.pbc[a];
    }
    g.PX = m.PX;
    const int gx = N[0] - 1 - d.pbc[0], gy = N[1] - 1 - d.pbc[1], gz = N[2] - 1 - d.pbc[2];
    int* dmap = nullptr;
    float* stage = nullptr;
    try {
        if (m.raster_bulk) {
            const int mx = (int)m.raster_map.size() - 1;
            check(cudaMalloc(&dmap, m.raster_map.size() * sizeof(int)), "rasterisation");
            check(cudaMemcpyAsync(dmap, m.raster_map.data(), m.raster_map.size() * sizeof(int), cudaMemcpyHostToDevice, s),
                  "rasterisation");
            // planes in chunks of at most 256 MiB
            const long long plane = (long long)gx * gy;
            const int chunk = (int)std::max<long long>(1, std::min<long long>(gz, (256LL << 20) / (plane * 4)));
            check(cudaMalloc(&stage, (size_t)chunk * plane * sizeof(float)), "rasterisation");
            for (int k0 = 0; k0 < gz; k0 += chunk) {
                const int nk = std::min(chunk, gz - k0);
                const size_t bytes = (size_t)nk * plane * sizeof(float);
                check(cudaMemcpyAsync(stage, m.raster_bulk + (size_t)k0 * plane, bytes, cudaMemcpyHostToDevice, s),
                      "bulk geometry upload");
                h2d += bytes;
                const long long n = (long long)nk * plane;
                const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 32);
                k_bulk_ids<<<blocks, 256, 0, s>>>(g, stage, gx, gy, k0, nk, dmap, mx, cell);
                check(cudaGetLastError(), "k_bulk_ids");
            }
        }
        int mid = 0;
        for (const Object& o : d.objects) {
            for (size_t r = 0; r < d.mats.size(); r++)
                if ((float)o.mat == d.mats[r].id) mid = (int)r + 1;
            ObjDev od{};
            od.mid = mid;
            for (int a = 0; a < 3; a++) od.a[a] = o.a[a];
            if (o.kind == Object::Block) {
                od.kind = 0;
                for (int a = 0; a < 3; a++) { od.lo[a] = o.a[a]; od.hi[a] = o.a[a] + o.b[a] - 1; }
            } else if (o.kind == Object::Sphere) {
                od.kind = 1;
                od.r = o.b[0];
                for (int a = 0; a < 3; a++) { od.lo[a] = o.a[a] - o.b[0]; od.hi[a] = o.a[a] + o.b[0] - 1; }
            } else {
                if (o.axis < 0) continue;
                od.kind = 2;
                od.r = o.b[1];
                od.axis = o.axis;
                for (int a = 0; a < 3; a++) {
                    if (a == o.axis) { od.lo[a] = o.a[a]; od.hi[a] = o.a[a] + o.b[0] - 1; }
                    else { od.lo[a] = o.a[a] - o.b[1]; od.hi[a] = o.a[a] + o.b[1] - 1; }
                }
            }
            // cells outside 1..N-1 are never written: clip the box
            bool empty = false;
            for (int a = 0; a < 3; a++) {
                od.lo[a] = std::max(od.lo[a], 1);
                od.hi[a] = std::min(od.hi[a], N[a] - 1);
                if (od.hi[a] < od.lo[a]) empty = true;
            }
            if (empty) continue;
            const long long n = (long long)(od.hi[0] - od.lo[0] + 1) * (od.hi[1] - od.lo[1] + 1) * (od.hi[2] - od.lo[2] + 1);
            const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 32);
            k_object_ids<<<blocks, 256, 0, s>>>(g, od, cell);
            check(cudaGetLastError(), "k_object_ids");
        }
        check(cudaStreamSynchronize(s), "rasterisation");
    } catch (...) {
        cudaFree(dmap);
        cudaFree(stage);
        throw;
    }
    cudaFree(dmap);
    cudaFree(stage);
}

}  // namespace aem
