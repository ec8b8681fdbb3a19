// nl.cu — cylinder neighbor list and boundary neighbor list on the device,
// with on-device re-vectorization of the excluded-volume and boundary force
// fields.
//
// Pair rule (HybridCylinderCylinderNL::updateNeighborsbin,
// src/Structure/HybridNeighborListImpl.cpp:332-471): a pair (c, n) is stored
// under the key cylinder c when c.id > n.id, the two are not on the same
// filament within |dposition| <= 2, and rmin^2 <= d^2 <= rmax^2, where d^2 is
// the squared distance of the midpoints 0.5*(b1 + b2) (Cylinder.cpp:48)
// summed x, y, z (Util/Math/Vec.hpp:378-384) and rmax^2, rmin^2 are float
// products (HybridNeighborListImpl.h:88-89). The bin grid is the reference's
// (bins of 1.125*sqrt(float rmax^2), HybridNeighborListImpl.cpp:176-240), so a
// midpoint outside it is the same error (getBin throws, :243-262). d^2 is
// rounded without contraction (__dmul_rn/__dadd_rn) so the pair set is the
// oracle's bit for bit.
//
// Passes: midpoints + bin index -> bin counts -> scan -> scatter -> sort each
// bin by cylinder index (deterministic order) -> per-key neighbor counts
// (27-bin stencil) -> scan -> write pairs / excluded-volume records, and
// per-plane boundary terms. One host synchronization reads the totals to size
// the outputs.
#include <algorithm>
#include <cstring>
#include <vector>

#include "handle.h"

namespace mb {

namespace {

constexpr int kScanBlock = 1024;

struct Grid {
    double bin;
    int g[3];
    double lim[3];  // bin * g, the exclusive upper bound of the grid
};

Grid make_grid(const medyan_nl_params& p) {
    Grid G{};
    const float rmaxsq = p.rmax * p.rmax;
    G.bin = 1.125 * (double)std::sqrt(rmaxsq);
    for (int d = 0; d < 3; ++d) {
        int size = (int)(p.grid_size[d]);
        int ib = (int)G.bin;
        G.g[d] = (ib != 0 && size % ib == 0) ? (int)(size / G.bin) : (int)(size / G.bin + 1);
        if (G.g[d] < 1) G.g[d] = 1;
        G.lim[d] = G.bin * G.g[d];
    }
    return G;
}

struct CylDev {
    int n;
    const int* b1;
    const int* b2;
    const int* id;
    const int* fil;
    const int* pos;
    const int* type;
    const int* branching;
    const int* minus_end;
    const double* eqlen;
    const double* exclk;
};

__global__ void k_midpoints(CylDev c, const double* __restrict__ x, Grid G, double* __restrict__ mid,
                            int* __restrict__ cell, int* __restrict__ bin_count, int* __restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const double* p1 = x + 3 * (size_t)c.b1[i];
    const double* p2 = x + 3 * (size_t)c.b2[i];
    long long idx = 0, stride = 1;
    bool bad = false;
    for (int d = 0; d < 3; ++d) {
        double m = 0.5 * (p1[d] + p2[d]);
        mid[3 * (size_t)i + d] = m;
        if (!(m >= 0.0) || m >= G.lim[d]) bad = true;
        int q = bad ? 0 : (int)(m / G.bin);
        idx += (long long)q * stride;
        stride *= G.g[d];
    }
    if (bad) {
        atomicOr(err, 1);
        cell[i] = -1;
        return;
    }
    cell[i] = (int)idx;
    atomicAdd(bin_count + idx, 1);
}

// Three-phase exclusive scan of int counts (in place into out[0..n], out[n] = total).
__global__ void k_scan_blocks(const int* __restrict__ in, int n, int* __restrict__ out, int* __restrict__ sums) {
    __shared__ int s[kScanBlock];
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    int v = i < n ? in[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kScanBlock; o <<= 1) {
        int t = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < n) out[i] = s[threadIdx.x] - v;
    if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = s[threadIdx.x];
}
__global__ void k_scan_sums(int* __restrict__ sums, int nb, int* __restrict__ total) {
    // one block: sequential chunks of kScanBlock
    __shared__ int s[kScanBlock];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += kScanBlock) {
        const int i = base + threadIdx.x;
        int v = i < nb ? sums[i] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < kScanBlock; o <<= 1) {
            int t = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < nb) sums[i] = s[threadIdx.x] - v + carry;
        __syncthreads();
        if (threadIdx.x == kScanBlock - 1) carry += s[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}
__global__ void k_scan_add(int* __restrict__ out, int n, const int* __restrict__ sums, const int* __restrict__ total) {
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
    if (i == 0) out[n] = *total;
}

__global__ void k_scatter(int n, const int* __restrict__ cell, const int* __restrict__ start, int* __restrict__ fillc,
                          int* __restrict__ items) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || cell[i] < 0) return;
    int slot = atomicAdd(fillc + cell[i], 1);
    items[start[cell[i]] + slot] = i;
}

// Deterministic bin contents: each bin sorted by cylinder index.
__global__ void k_sort_bins(int nbins, const int* __restrict__ start, int* __restrict__ items) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbins) return;
    const int s0 = start[b], s1 = start[b + 1];
    for (int a = s0 + 1; a < s1; ++a) {
        int v = items[a], q = a - 1;
        while (q >= s0 && items[q] > v) {
            items[q + 1] = items[q];
            --q;
        }
        items[q + 1] = v;
    }
}

// d^2 of the midpoints, rounded as written: ((dx*dx + dy*dy) + dz*dz).
__device__ __forceinline__ double dist2(const double* __restrict__ mid, int i, int j) {
    double dx = __dadd_rn(mid[3 * (size_t)j], -mid[3 * (size_t)i]);
    double dy = __dadd_rn(mid[3 * (size_t)j + 1], -mid[3 * (size_t)i + 1]);
    double dz = __dadd_rn(mid[3 * (size_t)j + 2], -mid[3 * (size_t)i + 2]);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// mode 0: count pairs per key; mode 1: write pairs (key, neighbor) for the
// standalone build; mode 2: write excluded-volume records (branch-parent pairs
// skipped, CylinderExclVolume.cpp:85).
template <int MODE>
__global__ void k_pairs(CylDev c, Grid G, const double* __restrict__ mid, const int* __restrict__ cell,
                        const int* __restrict__ start, const int* __restrict__ items, double rmaxsq, double rminsq,
                        int skip_branch, int* __restrict__ count, const int* __restrict__ offset,
                        int2* __restrict__ pairs, int4* __restrict__ ex_bs, double* __restrict__ ex_krs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n || cell[i] < 0) return;
    const int ci = cell[i];
    const int ix = ci % G.g[0], iy = (ci / G.g[0]) % G.g[1], iz = ci / (G.g[0] * G.g[1]);
    const int idi = c.id[i], fi = c.fil[i], pi = c.pos[i];
    int n = 0;
    int out = MODE == 0 ? 0 : offset[i];
    for (int dx = -1; dx <= 1; ++dx) {
        const int jx = ix + dx;
        if (jx < 0 || jx >= G.g[0]) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int jy = iy + dy;
            if (jy < 0 || jy >= G.g[1]) continue;
            for (int dz = -1; dz <= 1; ++dz) {
                const int jz = iz + dz;
                if (jz < 0 || jz >= G.g[2]) continue;
                const int cj = jx + G.g[0] * (jy + G.g[1] * jz);
                for (int q = start[cj]; q < start[cj + 1]; ++q) {
                    const int j = items[q];
                    if (idi <= c.id[j]) continue;
                    if (fi == c.fil[j]) {
                        int ds = pi - c.pos[j];
                        if ((ds < 0 ? -ds : ds) <= 2) continue;
                    }
                    const double d2 = dist2(mid, i, j);
                    if (d2 > rmaxsq || d2 < rminsq) continue;
                    if (skip_branch && c.branching[j] == i) continue;
                    if (MODE == 1) pairs[out + n] = make_int2(i, j);
                    if (MODE == 2) {
                        ex_bs[out + n] = make_int4(3 * c.b1[i], 3 * c.b2[i], 3 * c.b1[j], 3 * c.b2[j]);
                        double k = c.exclk[i];
                        if (c.type[i] != c.type[j]) k = k < c.exclk[j] ? c.exclk[j] : k;
                        ex_krs[out + n] = k * c.eqlen[i] * c.eqlen[j];
                    }
                    ++n;
                }
            }
        }
    }
    if (MODE == 0) count[i] = n;
}

// Canonical order for the standalone build: each key's neighbors ascending.
__global__ void k_sort_pairs(int n, const int* __restrict__ offset, int2* __restrict__ pairs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s0 = offset[i], s1 = offset[i + 1];
    for (int a = s0 + 1; a < s1; ++a) {
        int2 v = pairs[a];
        int q = a - 1;
        while (q >= s0 && pairs[q].y > v.y) {
            pairs[q + 1] = pairs[q];
            --q;
        }
        pairs[q + 1] = v;
    }
}

// Boundary NL: number of terms of cylinder i against plane p (0, 1 or 2).
__device__ __forceinline__ int boundary_terms(const CylDev& c, const double* __restrict__ x, const double4& pl,
                                              float cutoff, int i) {
    const double* p1 = x + 3 * (size_t)c.b1[i];
    const double* p2 = x + 3 * (size_t)c.b2[i];
    // Cylinder::coordinate = midPointCoordinate(b1, b2, 0.5) (Cylinder.cpp:46)
    double m[3];
    for (int d = 0; d < 3; ++d) m[d] = p1[d] * (1.0 - 0.5) + 0.5 * p2[d];
    double dist = (pl.x * m[0] + pl.y * m[1] + pl.z * m[2] + pl.w) / sqrt(pl.x * pl.x + pl.y * pl.y + pl.z * pl.z);
    if (!(dist < (double)cutoff)) return 0;
    return (c.minus_end && c.minus_end[i]) ? 2 : 1;
}
__global__ void k_boundary_count(CylDev c, const double* __restrict__ x, const double4* __restrict__ planes,
                                 int n_planes, float cutoff, int* __restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    for (int p = 0; p < n_planes; ++p) count[(size_t)p * c.n + i] = boundary_terms(c, x, planes[p], cutoff, i);
}
__global__ void k_boundary_write(CylDev c, const double* __restrict__ x, const double4* __restrict__ planes,
                                 int n_planes, float cutoff, double k, double slen, const int* __restrict__ offset,
                                 int* __restrict__ bs, double2* __restrict__ bp, int* __restrict__ bplane) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    for (int p = 0; p < n_planes; ++p) {
        int t = boundary_terms(c, x, planes[p], cutoff, i);
        if (!t) continue;
        int o = offset[(size_t)p * c.n + i];
        if (t == 2) {
            bs[o] = 3 * c.b1[i];
            bp[o] = make_double2(k, slen);
            bplane[o] = p;
            ++o;
        }
        bs[o] = 3 * c.b2[i];
        bp[o] = make_double2(k, slen);
        bplane[o] = p;
    }
}

// BoundaryCylinderRepulsion::computeLoadForces with the exponential
// repulsion (BoundaryCylinderRepulsion.cpp:125-196, BoundaryCylinderRepulsionExp.cpp:113-118):
// one block per tip, threads over the tip's monomer positions; planes in
// order, each plane whose neighbor list (member[p*n + cyl] > 0, from the last
// build) holds the tip's cylinder adds its term.
__global__ void k_boundary_load(CylDev c, const double* __restrict__ x, const double4* __restrict__ planes,
                                int n_planes, const int* __restrict__ member, double k, double slen, int n_tips,
                                const int* __restrict__ tip_cyl, const int* __restrict__ tip_plus,
                                const int* __restrict__ tip_nmon, const double* __restrict__ tip_mon,
                                const long long* __restrict__ tip_off, double* __restrict__ out) {
    for (int t = blockIdx.x; t < n_tips; t += gridDim.x) {
        const int ci = tip_cyl[t];
        const bool plus = tip_plus[t] != 0;
        const double* bo = x + 3 * (size_t)(plus ? c.b1[ci] : c.b2[ci]);
        const double* bd = x + 3 * (size_t)(plus ? c.b2[ci] : c.b1[ci]);
        // normalizedVector(bd - bo)
        const double vx = bd[0] - bo[0], vy = bd[1] - bo[1], vz = bd[2] - bo[2];
        const double m = sqrt(vx * vx + vy * vy + vz * vz);
        const double dir[3] = {vx / m, vy / m, vz / m};
        const int nmon = tip_nmon[t];
        const double mon = tip_mon[t];
        double* o = out + tip_off[t];
        for (int i = threadIdx.x; i < nmon; i += blockDim.x) {
            const double s = i * mon;
            const double p[3] = {bd[0] + s * dir[0], bd[1] + s * dir[1], bd[2] + s * dir[2]};
            double load = 0.0;
            for (int q = 0; q < n_planes; ++q) {
                if (member[(size_t)q * c.n + ci] <= 0) continue;
                const double4 pl = planes[q];
                const double proj0 = -(pl.x * dir[0] + pl.y * dir[1] + pl.z * dir[2]);
                const double proj = proj0 < 0.0 ? 0.0 : proj0;  // std::max(.., 0.0)
                const double dist =
                    (pl.x * p[0] + pl.y * p[1] + pl.z * p[2] + pl.w) / sqrt(pl.x * pl.x + pl.y * pl.y + pl.z * pl.z);
                const double R = -dist / slen;
                load += proj * (k * exp(R) / slen);
            }
            o[i] = load;
        }
    }
}

}  // namespace

// Device buffers of one neighbor-list builder (grow-only).
struct NLBuilder {
    DevBuf<int> b1, b2, id, fil, pos, type, branching, minus_end;
    DevBuf<double> eqlen, exclk;
    DevBuf<double> mid;
    DevBuf<int> cell, bin_count, bin_start, bin_fill, items, pair_count, pair_off, scan_sums, totals, err;
    DevBuf<int> bcount, boff;
    DevBuf<int2> pairs;
    DevBuf<double4> planes;
    medyan_nl_params nl{};
    medyan_boundary_params bp{};
    std::vector<double> plane_host;
    bool has_boundary = false;
    bool boundary_built = false;  // bcount holds the last build's plane membership
    int n = 0;

    CylDev view() const {
        return CylDev{n, b1.raw(), b2.raw(), id.raw(), fil.raw(), pos.raw(), type.raw(), branching.raw(),
                      minus_end.raw(), eqlen.raw(), exclk.raw()};
    }

    cudaError_t set(const medyan_cylinders* c, cudaStream_t s) {
        n = c->n_cyl;
        boundary_built = false;
        std::vector<int> zeros(n, 0), neg(n, -1);
        std::vector<double> dz(n, 0.0);
        cudaError_t e;
#define SETI(buf, ptr, dflt)                                                \
    e = (buf).assign((ptr) ? (ptr) : dflt.data(), (size_t)n, s);           \
    if (e != cudaSuccess) return e;
        SETI(b1, c->bead1, zeros);
        SETI(b2, c->bead2, zeros);
        SETI(id, c->id, zeros);
        SETI(fil, c->filament_id, zeros);
        SETI(pos, c->position_on_filament, zeros);
        SETI(type, c->type, zeros);
        SETI(branching, c->branching_cylinder, neg);
        SETI(minus_end, c->is_minus_end, zeros);
        SETI(eqlen, c->eq_length, dz);
        SETI(exclk, c->excl_k, dz);
#undef SETI
        return cudaSuccess;
    }

    // scan of cnt[0..m) into off[0..m] (off[m] = total)
    cudaError_t scan(const int* cnt, int m, int* off, cudaStream_t s) {
        const int nb = (m + kScanBlock - 1) / kScanBlock;
        cudaError_t e = scan_sums.reserve(nb + 1);
        if (e == cudaSuccess) e = totals.reserve(4);
        if (e != cudaSuccess) return e;
        if (m == 0) return cudaMemsetAsync(off, 0, sizeof(int), s);
        k_scan_blocks<<<nb, kScanBlock, 0, s>>>(cnt, m, off, scan_sums.raw());
        k_scan_sums<<<1, kScanBlock, 0, s>>>(scan_sums.raw(), nb, totals.raw());
        k_scan_add<<<nb, kScanBlock, 0, s>>>(off, m, scan_sums.raw(), totals.raw());
        return cudaGetLastError();
    }

    // Bins the midpoints and counts pairs per key; returns the pair total.
    medyan_status count_pairs(const double* x, int skip_branch, cudaStream_t s, long long* total) {
        const Grid G = make_grid(nl);
        const long long nbins = (long long)G.g[0] * G.g[1] * G.g[2];
        if (nbins > (1LL << 30)) return MEDYAN_ERR_INVALID_ARG;
        cudaError_t e = mid.reserve(3 * (size_t)std::max(n, 1));
        if (e == cudaSuccess) e = cell.reserve(std::max(n, 1));
        if (e == cudaSuccess) e = items.reserve(std::max(n, 1));
        if (e == cudaSuccess) e = bin_count.reserve(nbins + 1);
        if (e == cudaSuccess) e = bin_start.reserve(nbins + 1);
        if (e == cudaSuccess) e = bin_fill.reserve(nbins + 1);
        if (e == cudaSuccess) e = pair_count.reserve(n + 1);
        if (e == cudaSuccess) e = pair_off.reserve(n + 1);
        if (e == cudaSuccess) e = err.reserve(1);
        if (e != cudaSuccess) return cuda_status(e);
        cudaMemsetAsync(bin_count.raw(), 0, sizeof(int) * (nbins + 1), s);
        cudaMemsetAsync(bin_fill.raw(), 0, sizeof(int) * (nbins + 1), s);
        cudaMemsetAsync(err.raw(), 0, sizeof(int), s);
        const int tb = 256, gb = (n + tb - 1) / tb;
        if (n > 0) k_midpoints<<<gb, tb, 0, s>>>(view(), x, G, mid.raw(), cell.raw(), bin_count.raw(), err.raw());
        e = scan(bin_count.raw(), (int)nbins, bin_start.raw(), s);
        if (e != cudaSuccess) return cuda_status(e);
        if (n > 0) {
            k_scatter<<<gb, tb, 0, s>>>(n, cell.raw(), bin_start.raw(), bin_fill.raw(), items.raw());
            k_sort_bins<<<(int)((nbins + tb - 1) / tb), tb, 0, s>>>((int)nbins, bin_start.raw(), items.raw());
            const float rmaxsq = nl.rmax * nl.rmax, rminsq = nl.rmin * nl.rmin;
            k_pairs<0><<<gb, tb, 0, s>>>(view(), G, mid.raw(), cell.raw(), bin_start.raw(), items.raw(),
                                         (double)rmaxsq, (double)rminsq, skip_branch, pair_count.raw(), nullptr,
                                         nullptr, nullptr, nullptr);
        }
        e = scan(pair_count.raw(), n, pair_off.raw(), s);
        if (e != cudaSuccess) return cuda_status(e);
        int h[2] = {0, 0};
        e = cudaMemcpyAsync(&h[0], pair_off.raw() + n, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h[1], err.raw(), sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e);
        if (h[1]) return MEDYAN_ERR_OUT_OF_GRID;
        *total = h[0];
        return MEDYAN_OK;
    }

    template <int MODE>
    void write_pairs(const double* x, int skip_branch, int2* out_pairs, int4* ex_bs, double* ex_krs, cudaStream_t s) {
        (void)x;
        const Grid G = make_grid(nl);
        const int tb = 256, gb = (n + tb - 1) / tb;
        if (n == 0) return;
        const float rmaxsq = nl.rmax * nl.rmax, rminsq = nl.rmin * nl.rmin;
        k_pairs<MODE><<<gb, tb, 0, s>>>(view(), G, mid.raw(), cell.raw(), bin_start.raw(), items.raw(),
                                        (double)rmaxsq, (double)rminsq, skip_branch, nullptr, pair_off.raw(),
                                        out_pairs, ex_bs, ex_krs);
        if (MODE == 1) k_sort_pairs<<<gb, tb, 0, s>>>(n, pair_off.raw(), out_pairs);
    }

    // Boundary NL + vectorization into the handle's boundary records.
    medyan_status boundary(medyan_mech* h, const double* x, cudaStream_t s, long long* total) {
        *total = 0;
        if (!has_boundary || bp.n_planes <= 0) return MEDYAN_OK;
        const int np = bp.n_planes;
        cudaError_t e = bcount.reserve((size_t)np * n + 1);
        if (e == cudaSuccess) e = boff.reserve((size_t)np * n + 1);
        if (e != cudaSuccess) return cuda_status(e);
        const int tb = 256, gb = (n + tb - 1) / tb;
        if (n > 0) k_boundary_count<<<gb, tb, 0, s>>>(view(), x, planes.raw(), np, bp.cutoff, bcount.raw());
        e = scan(bcount.raw(), np * n, boff.raw(), s);
        if (e != cudaSuccess) return cuda_status(e);
        int tot = 0;
        e = cudaMemcpyAsync(&tot, boff.raw() + (size_t)np * n, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess) e = h->boundary_bs.reserve(tot);
        if (e == cudaSuccess) e = h->boundary_p.reserve(tot);
        if (e == cudaSuccess) e = h->boundary_plane.reserve(tot);
        if (e == cudaSuccess) e = h->planes.assign(planes_host4().data(), np, s);
        if (e != cudaSuccess) return cuda_status(e);
        if (n > 0 && tot > 0)
            k_boundary_write<<<gb, tb, 0, s>>>(view(), x, planes.raw(), np, bp.cutoff, bp.k, bp.screen_length,
                                               boff.raw(), h->boundary_bs.raw(), h->boundary_p.raw(),
                                               h->boundary_plane.raw());
        h->ff.n_boundary = tot;
        h->ff.n_planes = np;
        *total = tot;
        e = cudaGetLastError();
        boundary_built = e == cudaSuccess;
        return cuda_status(e);
    }

    std::vector<double4> planes_host4() const {
        std::vector<double4> v(bp.n_planes);
        for (int p = 0; p < bp.n_planes; ++p)
            v[p] = make_double4(plane_host[4 * p], plane_host[4 * p + 1], plane_host[4 * p + 2], plane_host[4 * p + 3]);
        return v;
    }
};

void destroy_nl(medyan_mech* h) {
    delete reinterpret_cast<NLBuilder*>(h->nl);
    h->nl = nullptr;
}

}  // namespace mb

using namespace mb;

extern "C" {

medyan_status medyan_nl_build(const medyan_cylinders* cyl, const double* coord, int32_t n_beads,
                              const medyan_nl_params* p, int32_t* pairs_out, int64_t capacity, int64_t* n_pairs) {
    if (!cyl || !p || !n_pairs || cyl->n_cyl < 0 || n_beads < 0 || (!coord && n_beads)) return MEDYAN_ERR_INVALID_ARG;
    if (!(p->rmax > 0) || p->rmin < 0) return MEDYAN_ERR_INVALID_ARG;
    for (int i = 0; i < cyl->n_cyl; ++i) {
        if (!cyl->bead1 || !cyl->bead2 || !cyl->id || !cyl->filament_id || !cyl->position_on_filament)
            return MEDYAN_ERR_INVALID_ARG;
        if (cyl->bead1[i] < 0 || cyl->bead1[i] >= n_beads || cyl->bead2[i] < 0 || cyl->bead2[i] >= n_beads)
            return MEDYAN_ERR_INDEX_RANGE;
    }
    cudaStream_t s;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_status(e);
    medyan_status st = MEDYAN_OK;
    {
        NLBuilder b;
        b.nl = *p;
        DevBuf<double> x;
        e = b.set(cyl, s);
        if (e == cudaSuccess) e = x.assign(coord, 3 * (size_t)n_beads, s);
        if (e != cudaSuccess) st = cuda_status(e);
        long long total = 0;
        if (st == MEDYAN_OK) st = b.count_pairs(x.raw(), 0, s, &total);
        if (st == MEDYAN_OK) {
            *n_pairs = total;
            if (pairs_out) {
                if (total > capacity) st = MEDYAN_ERR_CAPACITY;
                else if (total > 0) {
                    e = b.pairs.reserve(total);
                    if (e == cudaSuccess) {
                        b.write_pairs<1>(x.raw(), 0, b.pairs.raw(), nullptr, nullptr, s);
                        e = cudaMemcpyAsync(pairs_out, b.pairs.raw(), sizeof(int2) * total, cudaMemcpyDeviceToHost, s);
                    }
                    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                    if (e != cudaSuccess) st = cuda_status(e);
                }
            }
        } else {
            *n_pairs = 0;
        }
        cudaStreamSynchronize(s);
    }
    cudaStreamDestroy(s);
    return st;
}

medyan_status medyan_mech_set_cylinders(medyan_mech* h, const medyan_cylinders* cyl, const medyan_nl_params* nl,
                                        const medyan_boundary_params* boundary) {
    if (!h || !cyl || !nl || cyl->n_cyl < 0 || !(nl->rmax > 0) || nl->rmin < 0) return MEDYAN_ERR_INVALID_ARG;
    if (!cyl->bead1 || !cyl->bead2 || !cyl->id || !cyl->filament_id || !cyl->position_on_filament || !cyl->eq_length ||
        !cyl->excl_k)
        return MEDYAN_ERR_INVALID_ARG;
    for (int i = 0; i < cyl->n_cyl; ++i) {
        if (cyl->bead1[i] < 0 || cyl->bead1[i] >= h->n_beads || cyl->bead2[i] < 0 || cyl->bead2[i] >= h->n_beads)
            return MEDYAN_ERR_INDEX_RANGE;
        if (cyl->branching_cylinder && (cyl->branching_cylinder[i] < -1 || cyl->branching_cylinder[i] >= cyl->n_cyl))
            return MEDYAN_ERR_INDEX_RANGE;
    }
    if (boundary && boundary->n_planes > 0 && !boundary->plane_eq) return MEDYAN_ERR_INVALID_ARG;
    if (!h->nl) h->nl = reinterpret_cast<medyan_mech::NL*>(new NLBuilder());
    NLBuilder* b = reinterpret_cast<NLBuilder*>(h->nl);
    b->nl = *nl;
    b->has_boundary = boundary && boundary->n_planes > 0;
    if (b->has_boundary) {
        b->bp = *boundary;
        b->plane_host.assign(boundary->plane_eq, boundary->plane_eq + 4 * boundary->n_planes);
        b->bp.plane_eq = b->plane_host.data();
        cudaError_t e = b->planes.assign(b->planes_host4().data(), boundary->n_planes, h->stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    // bead indices into the handle's internal order
    std::vector<int32_t> b1(cyl->n_cyl), b2(cyl->n_cyl);
    for (int i = 0; i < cyl->n_cyl; ++i) {
        b1[i] = h->pos_host.empty() ? cyl->bead1[i] : h->pos_host[cyl->bead1[i]];
        b2[i] = h->pos_host.empty() ? cyl->bead2[i] : h->pos_host[cyl->bead2[i]];
    }
    medyan_cylinders ci = *cyl;
    ci.bead1 = b1.data();
    ci.bead2 = b2.data();
    cudaError_t e = b->set(&ci, h->stream);
    return cuda_status(e);
}

medyan_status medyan_mech_rebuild_neighbors(medyan_mech* h, int64_t* n_excl_out, int64_t* n_boundary_out) {
    if (!h || !h->nl) return MEDYAN_ERR_INVALID_ARG;
    NLBuilder* b = reinterpret_cast<NLBuilder*>(h->nl);
    cudaStream_t s = h->stream;
    long long total = 0;
    medyan_status st = b->count_pairs(h->x.raw(), 1, s, &total);
    if (st != MEDYAN_OK) return st;
    cudaError_t e = h->excl_bs.reserve(total);
    if (e == cudaSuccess) e = h->excl_krs.reserve(total);
    if (e != cudaSuccess) return cuda_status(e);
    b->write_pairs<2>(h->x.raw(), 1, nullptr, h->excl_bs.raw(), h->excl_krs.raw(), s);
    h->ff.n_excl = (int)total;
    long long nb = 0;
    st = b->boundary(h, h->x.raw(), s, &nb);
    if (st != MEDYAN_OK) return st;
    st = refresh_device_ff(h);
    if (st != MEDYAN_OK) return st;
    if (n_excl_out) *n_excl_out = total;
    if (n_boundary_out) *n_boundary_out = nb;
    return sync_status(h);
}

medyan_status medyan_mech_get_excl_volume(medyan_mech* h, int32_t* beads_out, double* k_out, double* eqlen_out,
                                          int64_t capacity, int64_t* n_out) {
    if (!h || !n_out) return MEDYAN_ERR_INVALID_ARG;
    const int64_t n = h->ff.n_excl;
    *n_out = n;
    if (!beads_out) return MEDYAN_OK;
    if (n > capacity) return MEDYAN_ERR_CAPACITY;
    if (n == 0) return MEDYAN_OK;
    std::vector<int4> bs(n);
    std::vector<double> krs(n);
    cudaError_t e = cudaMemcpyAsync(bs.data(), h->excl_bs.raw(), sizeof(int4) * n, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(krs.data(), h->excl_krs.raw(), sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_status(e);
    // internal offsets back to the caller's bead order
    auto ext = [&](int off) { return h->order_host.empty() ? off : 3 * h->order_host[off / 3]; };
    for (int64_t i = 0; i < n; ++i) {
        beads_out[4 * i] = ext(bs[i].x);
        beads_out[4 * i + 1] = ext(bs[i].y);
        beads_out[4 * i + 2] = ext(bs[i].z);
        beads_out[4 * i + 3] = ext(bs[i].w);
        // the device keeps krep*L1*L2; report it with unit lengths
        if (k_out) k_out[i] = krs[i];
        if (eqlen_out) {
            eqlen_out[2 * i] = 1.0;
            eqlen_out[2 * i + 1] = 1.0;
        }
    }
    return MEDYAN_OK;
}

}  // extern "C"

extern "C" medyan_status medyan_mech_boundary_load_forces(medyan_mech* h, const medyan_load_tips* tips,
                                                          double* load_out, int64_t capacity) {
    if (!h || !tips || tips->n_tips < 0) return MEDYAN_ERR_INVALID_ARG;
    const int nt = tips->n_tips;
    if (nt == 0) return MEDYAN_OK;
    if (!tips->cylinder || !tips->plus_end || !tips->n_mon || !tips->mon_size || !load_out)
        return MEDYAN_ERR_INVALID_ARG;
    NLBuilder* b = reinterpret_cast<NLBuilder*>(h->nl);
    if (!b) return MEDYAN_ERR_INVALID_ARG;  // no cylinder list: medyan_mech_set_cylinders first
    std::vector<long long> off(nt);
    long long tot = 0;
    for (int t = 0; t < nt; ++t) {
        if (tips->n_mon[t] < 0 || tips->cylinder[t] < 0 || tips->cylinder[t] >= b->n) return MEDYAN_ERR_INVALID_ARG;
        off[t] = tot;
        tot += tips->n_mon[t];
    }
    if (tot > capacity) return MEDYAN_ERR_CAPACITY;
    if (!b->has_boundary || b->bp.n_planes <= 0) {
        std::fill(load_out, load_out + tot, 0.0);
        return MEDYAN_OK;
    }
    if (!b->boundary_built) return MEDYAN_ERR_INVALID_ARG;  // medyan_mech_rebuild_neighbors first
    if (tot == 0) return MEDYAN_OK;
    cudaError_t e = cudaSetDevice(h->device);
    cudaStream_t s = h->stream;
    DevBuf<int> cyl, plus, nmon;
    DevBuf<double> mon, out;
    DevBuf<long long> doff;
    if (e == cudaSuccess) e = cyl.assign(tips->cylinder, nt, s);
    if (e == cudaSuccess) e = plus.assign(tips->plus_end, nt, s);
    if (e == cudaSuccess) e = nmon.assign(tips->n_mon, nt, s);
    if (e == cudaSuccess) e = mon.assign(tips->mon_size, nt, s);
    if (e == cudaSuccess) e = doff.assign(off.data(), nt, s);
    if (e == cudaSuccess) e = out.reserve(tot);
    if (e != cudaSuccess) return cuda_status(e);
    const int g = nt < 148 * 8 ? nt : 148 * 8;
    k_boundary_load<<<g, 128, 0, s>>>(b->view(), h->x.raw(), b->planes.raw(), b->bp.n_planes, b->bcount.raw(),
                                      b->bp.k, b->bp.screen_length, nt, cyl.raw(), plus.raw(), nmon.raw(),
                                      mon.raw(), doff.raw(), out.raw());
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(load_out, out.raw(), sizeof(double) * tot, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e);
}
