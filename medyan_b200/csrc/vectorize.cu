// vectorize.cu — the handle's device records built on the device from the
// caller's vectorized arrays (ForceFieldManager::vectorizeAllForceFields,
// ForceFieldManager.cpp:35-93, and each ForceField::vectorize).
//
// The caller's arrays (bead sets as coordinate offsets 3*bead, parameters per
// interaction) are copied to the device as they are, and kernels do what
// the host loops of upload_system (capi.cu) do, in the same order, so both
// produce the same records bit for bit:
//   - filament chains: link i (b1 -> b2) with pos[b2] == pos[b1] + 1 belongs
//     to the chain at position pos[b1], bend i (b1, b2, b3) with consecutive
//     positions to the chain at pos[b2]; when several fit one position, the
//     lowest index wins (an atomicMin claim), as the host's first-come order
//     gives;
//   - leftover links and bends: the rest, compacted in index order (a
//     prefix scan of the leftover flags), with their bead offsets in the
//     internal order;
//   - linker, motor, branch, excluded-volume and boundary records: the bead
//     offsets remapped to the internal order, the parameters packed per
//     record (kRS = k * L1 * L2 as the host forms it).
// The host keeps what is not per-record work: argument validation, the
// internal bead order (a walk of the links, once per bead count) and the
// counts that size the launches (two leftover counts read back).
#include <cstring>

#include "handle.h"

namespace mb {

namespace {

constexpr int kThreads = 256;
constexpr int kScanBlock = 1024;
constexpr unsigned char kLink = 1, kBend = 2;
constexpr int kNoOwner = 0x7f7f7f7f;  // the owners' fill (a byte memset): above every index

int grid_for(long long n) {
    const long long b = (n + kThreads - 1) / kThreads;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

#define GRID_STRIDE(i, n) \
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

// external coordinate offset -> internal one
__device__ __forceinline__ int remap(const int* __restrict__ pos, int off) { return 3 * pos[off / 3]; }

// Chain claims: the lowest interaction index that fits each position.
__global__ void k_claim(const int* __restrict__ pos, const int* __restrict__ sb, int ns, const int* __restrict__ bb,
                        int nbd, int* __restrict__ link_owner, int* __restrict__ bend_owner) {
    GRID_STRIDE(i, ns) {
        const int p = pos[sb[2 * i] / 3], q = pos[sb[2 * i + 1] / 3];
        if (q == p + 1) atomicMin(link_owner + p, i);
    }
    GRID_STRIDE(i, nbd) {
        const int p1 = pos[bb[3 * i] / 3], p = pos[bb[3 * i + 1] / 3], p3 = pos[bb[3 * i + 2] / 3];
        if (p1 == p - 1 && p3 == p + 1) atomicMin(bend_owner + p, i);
    }
}

// Per position: flags and the owning link's and bend's parameters.
__global__ void k_chain_fill(int n, const int* __restrict__ link_owner, const int* __restrict__ bend_owner,
                             const double* __restrict__ sk, const double* __restrict__ sl,
                             const double* __restrict__ bk, const double* __restrict__ bt,
                             unsigned char* __restrict__ flags, double2* __restrict__ link_p,
                             double2* __restrict__ bend_p) {
    GRID_STRIDE(p, n) {
        const int lo = link_owner[p], bo = bend_owner[p];
        unsigned char fl = 0;
        double2 lp = make_double2(0.0, 0.0), bp = make_double2(0.0, 0.0);
        if (lo != kNoOwner) {
            fl |= kLink;
            lp = make_double2(sk[lo], sl[lo]);
        }
        if (bo != kNoOwner) {
            fl |= kBend;
            bp = make_double2(bk[bo], bt[bo]);
        }
        flags[p] = fl;
        link_p[p] = lp;
        bend_p[p] = bp;
    }
}

// 1 for each link / bend that no chain took.
__global__ void k_left_flags(const int* __restrict__ pos, const int* __restrict__ sb, int ns,
                             const int* __restrict__ bb, int nbd, const int* __restrict__ link_owner,
                             const int* __restrict__ bend_owner, int* __restrict__ ls, int* __restrict__ lb) {
    GRID_STRIDE(i, ns) {
        const int p = pos[sb[2 * i] / 3], q = pos[sb[2 * i + 1] / 3];
        ls[i] = (q == p + 1 && link_owner[p] == i) ? 0 : 1;
    }
    GRID_STRIDE(i, nbd) {
        const int p1 = pos[bb[3 * i] / 3], p = pos[bb[3 * i + 1] / 3], p3 = pos[bb[3 * i + 2] / 3];
        lb[i] = (p1 == p - 1 && p3 == p + 1 && bend_owner[p] == i) ? 0 : 1;
    }
}

// Exclusive prefix sum of in[0, n) into out, and the total into *total: one
// block per kScanBlock elements, then the block sums (one thread, in order),
// then the add.
__global__ void __launch_bounds__(kScanBlock) k_scan_local(const int* __restrict__ in, int n, int* __restrict__ out,
                                                           int* __restrict__ sums) {
    __shared__ int s[kScanBlock];
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kScanBlock; o <<= 1) {
        const int t = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < n) out[i] = s[threadIdx.x] - v;
    if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = s[threadIdx.x];
}

__global__ void k_scan_block_sums(int* __restrict__ sums, int nb, int* __restrict__ total) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int acc = 0;
    for (int b = 0; b < nb; ++b) {
        const int v = sums[b];
        sums[b] = acc;
        acc += v;
    }
    *total = acc;
}

__global__ void k_scan_apply(int* __restrict__ out, int n, const int* __restrict__ sums) {
    GRID_STRIDE(i, n) out[i] += sums[i / kScanBlock];
}

// Leftover records in index order, and the caller's-index -> chain position
// or leftover record map of the parameter gradients.
__global__ void k_left_write(const int* __restrict__ pos, const int* __restrict__ sb, const double* __restrict__ sk,
                             const double* __restrict__ sl, int ns, const int* __restrict__ ls,
                             const int* __restrict__ ls_rank, const int* __restrict__ bb,
                             const double* __restrict__ bk, const double* __restrict__ bt, int nbd,
                             const int* __restrict__ lb, const int* __restrict__ lb_rank, int2* __restrict__ s_bs,
                             double2* __restrict__ s_p, int4* __restrict__ b_bs, double2* __restrict__ b_p,
                             int* __restrict__ smap, int* __restrict__ bmap) {
    GRID_STRIDE(i, ns) {
        const int p = pos[sb[2 * i] / 3];
        if (ls[i]) {
            const int q = ls_rank[i];
            s_bs[q] = make_int2(remap(pos, sb[2 * i]), remap(pos, sb[2 * i + 1]));
            s_p[q] = make_double2(sk[i], sl[i]);
            smap[i] = -1 - q;
        } else {
            smap[i] = p;
        }
    }
    GRID_STRIDE(i, nbd) {
        const int p = pos[bb[3 * i + 1] / 3];
        if (lb[i]) {
            const int q = lb_rank[i];
            b_bs[q] = make_int4(remap(pos, bb[3 * i]), remap(pos, bb[3 * i + 1]), remap(pos, bb[3 * i + 2]), 0);
            b_p[q] = make_double2(bk[i], bt[i]);
            bmap[i] = -1 - q;
        } else {
            bmap[i] = p;
        }
    }
}

// Two-bead-pair springs (linkers, motors): (k, l0, pos1, pos2).
__global__ void k_springs(const int* __restrict__ pos, const int* __restrict__ bs, const double* __restrict__ k,
                          const double* __restrict__ l0, const double* __restrict__ p1, const double* __restrict__ p2,
                          int n, int4* __restrict__ out_bs, double4* __restrict__ out_p) {
    GRID_STRIDE(i, n) {
        out_bs[i] = make_int4(remap(pos, bs[4 * i]), remap(pos, bs[4 * i + 1]), remap(pos, bs[4 * i + 2]),
                              remap(pos, bs[4 * i + 3]));
        out_p[i] = make_double4(k[i], l0[i], p1[i], p2[i]);
    }
}

__device__ __forceinline__ double at(const double* p, int i) { return p ? p[i] : 0.0; }

// Branch points: pa = (position, stretch k, stretch l0, bend k),
// pb = (bend theta0, dihedral k, position k, 0).
__global__ void k_branches(const int* __restrict__ pos, const int* __restrict__ bs, const double* __restrict__ bpos,
                           const double* sk, const double* sl, const double* bk, const double* bt, const double* dk,
                           const double* pk, int n, int4* __restrict__ out_bs, double4* __restrict__ pa,
                           double4* __restrict__ pb) {
    GRID_STRIDE(i, n) {
        out_bs[i] = make_int4(remap(pos, bs[4 * i]), remap(pos, bs[4 * i + 1]), remap(pos, bs[4 * i + 2]),
                              remap(pos, bs[4 * i + 3]));
        pa[i] = make_double4(bpos[i], at(sk, i), at(sl, i), at(bk, i));
        pb[i] = make_double4(at(bt, i), at(dk, i), at(pk, i), 0.0);
    }
}

// Excluded-volume pairs: kRS = krep * eqLength_1 * eqLength_2
// (CylinderExclVolRepulsion.cpp:355), multiplied left to right as the host does.
__global__ void k_excl(const int* __restrict__ pos, const int* __restrict__ bs, const double* __restrict__ k,
                       const double* __restrict__ eql, int n, int4* __restrict__ out_bs, double* __restrict__ krs) {
    GRID_STRIDE(i, n) {
        out_bs[i] = make_int4(remap(pos, bs[4 * i]), remap(pos, bs[4 * i + 1]), remap(pos, bs[4 * i + 2]),
                              remap(pos, bs[4 * i + 3]));
        krs[i] = k[i] * eql[2 * i] * eql[2 * i + 1];
    }
}

// Boundary terms: bead, (k, screening length), and the plane each term
// belongs to (plane p owns the next nneighbors[p] terms).
__global__ void k_boundary(const int* __restrict__ pos, const int* __restrict__ bs, const double* __restrict__ k,
                           const double* __restrict__ sl, int n, const int* __restrict__ nn, int n_planes,
                           const double* __restrict__ eq, int* __restrict__ out_bs, double2* __restrict__ out_p,
                           int* __restrict__ out_plane, double4* __restrict__ planes) {
    GRID_STRIDE(i, n) {
        out_bs[i] = remap(pos, bs[i]);
        out_p[i] = make_double2(k[i], sl[i]);
        int p = 0, end = nn[0];
        while (i >= end && p + 1 < n_planes) end += nn[++p];
        out_plane[i] = p;
    }
    GRID_STRIDE(p, n_planes) planes[p] = make_double4(eq[4 * p], eq[4 * p + 1], eq[4 * p + 2], eq[4 * p + 3]);
}

size_t rounded(size_t bytes) { return (bytes + 255) / 256 * 256; }

// Device staging of the caller's arrays: one allocation, 256-byte aligned
// slices, one copy per array.
struct Staging {
    unsigned char* base;
    size_t off;
    cudaStream_t s;
    cudaError_t e;
    template <class T>
    const T* put(const T* host, size_t count) {
        if (e != cudaSuccess || !host || count == 0) return nullptr;
        T* d = reinterpret_cast<T*>(base + off);
        e = cudaMemcpyAsync(d, host, sizeof(T) * count, cudaMemcpyHostToDevice, s);
        off += rounded(sizeof(T) * count);
        return d;
    }
    template <class T>
    T* take(size_t count) {
        T* d = reinterpret_cast<T*>(base + off);
        off += rounded(sizeof(T) * count);
        return d;
    }
};

}  // namespace

medyan_status upload_system_device(medyan_mech* h, const medyan_system* s) {
    cudaStream_t st = h->stream;
    DeviceFF& ff = h->ff;
    const int bonded_block = ff.bonded_block, excl_block = ff.excl_block;  // launch shapes survive an update
    ff = DeviceFF{};
    ff.bonded_block = bonded_block;
    ff.excl_block = excl_block;
    ff.n_beads = s->n_beads;
    cudaError_t e = cudaSuccess;

    // the internal bead order is fixed by the first vectorization (host walk)
    if ((int)h->order_host.size() != s->n_beads || (int)h->pos_dev.n != s->n_beads) {
        if ((int)h->order_host.size() != s->n_beads) {
            chain_order(s, h->order_host);
            h->pos_host.assign(s->n_beads, 0);
            h->identity_order = true;
            for (int p = 0; p < s->n_beads; ++p) {
                h->pos_host[h->order_host[p]] = p;
                if (h->order_host[p] != p) h->identity_order = false;
            }
            if (!h->identity_order) e = h->order.assign(h->order_host.data(), h->order_host.size(), st);
            if (e == cudaSuccess) e = h->stage.reserve(3 * (size_t)s->n_beads);
        }
        if (e == cudaSuccess) e = h->pos_dev.assign(h->pos_host.data(), h->pos_host.size(), st);
        if (e != cudaSuccess) return cuda_status(e);
    }
    const int nb = s->n_beads;
    const int ns = s->n_stretch, nbd = s->n_bend, nl = s->n_linker, nm = s->n_motor, nr = s->n_branch,
              ne = s->n_excl, nbo = s->n_boundary, np = s->n_planes;
    const int nmax = ns > nbd ? ns : nbd;
    const int nsums = nmax / kScanBlock + 1;

    // staging: the caller's arrays, then the scratch of the chain claims
    size_t need = 0;
    need += rounded(sizeof(int) * 2 * (size_t)ns) + 2 * rounded(sizeof(double) * ns);
    need += rounded(sizeof(int) * 3 * (size_t)nbd) + 2 * rounded(sizeof(double) * nbd);
    need += rounded(sizeof(int) * 4 * (size_t)nl) + 4 * rounded(sizeof(double) * nl);
    need += rounded(sizeof(int) * 4 * (size_t)nm) + 4 * rounded(sizeof(double) * nm);
    need += rounded(sizeof(int) * 4 * (size_t)nr) + 7 * rounded(sizeof(double) * nr);
    need += rounded(sizeof(int) * 4 * (size_t)ne) + rounded(sizeof(double) * ne) + rounded(sizeof(double) * 2 * ne);
    need += rounded(sizeof(int) * nbo) + 2 * rounded(sizeof(double) * nbo);
    need += rounded(sizeof(double) * 4 * (size_t)np) + rounded(sizeof(int) * np);
    need += 2 * rounded(sizeof(int) * (size_t)nb);     // link / bend owners
    need += 4 * rounded(sizeof(int) * (size_t)nmax);   // leftover flags and ranks
    need += 2 * rounded(sizeof(int) * (size_t)nsums) + rounded(2 * sizeof(int));
    e = h->vec_stage.reserve(need ? need : 1);
    if (e != cudaSuccess) return cuda_status(e);
    Staging S{h->vec_stage.raw(), 0, st, cudaSuccess};
    const int* d_sb = S.put(s->stretch_beads, 2 * (size_t)ns);
    const double* d_sk = S.put(s->stretch_k, ns);
    const double* d_sl = S.put(s->stretch_l0, ns);
    const int* d_bb = S.put(s->bend_beads, 3 * (size_t)nbd);
    const double* d_bk = S.put(s->bend_k, nbd);
    const double* d_bt = S.put(s->bend_theta0, nbd);
    const int* d_lb = S.put(s->linker_beads, 4 * (size_t)nl);
    const double* d_lk = S.put(s->linker_k, nl);
    const double* d_ll = S.put(s->linker_l0, nl);
    const double* d_l1 = S.put(s->linker_pos1, nl);
    const double* d_l2 = S.put(s->linker_pos2, nl);
    const int* d_mb = S.put(s->motor_beads, 4 * (size_t)nm);
    const double* d_mk = S.put(s->motor_k, nm);
    const double* d_ml = S.put(s->motor_l0, nm);
    const double* d_m1 = S.put(s->motor_pos1, nm);
    const double* d_m2 = S.put(s->motor_pos2, nm);
    const int* d_rb = S.put(s->branch_beads, 4 * (size_t)nr);
    const double* d_rp = S.put(s->branch_pos, nr);
    const double* d_rsk = S.put(s->branch_stretch_k, nr);
    const double* d_rsl = S.put(s->branch_stretch_l0, nr);
    const double* d_rbk = S.put(s->branch_bend_k, nr);
    const double* d_rbt = S.put(s->branch_bend_theta0, nr);
    const double* d_rdk = S.put(s->branch_dihedral_k, nr);
    const double* d_rpk = S.put(s->branch_position_k, nr);
    const int* d_eb = S.put(s->excl_beads, 4 * (size_t)ne);
    const double* d_ek = S.put(s->excl_k, ne);
    const double* d_el = S.put(s->excl_eqlen, 2 * (size_t)ne);
    const int* d_ob = S.put(s->boundary_beads, nbo);
    const double* d_ok = S.put(s->boundary_k, nbo);
    const double* d_os = S.put(s->boundary_slen, nbo);
    const double* d_pe = S.put(s->plane_eq, 4 * (size_t)np);
    const int* d_pn = S.put(s->plane_nneighbors, np);
    if (S.e != cudaSuccess) return cuda_status(S.e);
    int* link_owner = S.take<int>(nb);
    int* bend_owner = S.take<int>(nb);
    int* ls = S.take<int>(nmax);
    int* lb = S.take<int>(nmax);
    int* ls_rank = S.take<int>(nmax);
    int* lb_rank = S.take<int>(nmax);
    int* sums_s = S.take<int>(nsums);
    int* sums_b = S.take<int>(nsums);
    int* totals = S.take<int>(2);
    const int* pos = h->pos_dev.raw();

    // filament chains
    e = h->chain_flags.reserve(nb);
    if (e == cudaSuccess) e = h->chain_link_p.reserve(nb);
    if (e == cudaSuccess) e = h->chain_bend_p.reserve(nb);
    if (e == cudaSuccess) e = h->stretch_map.reserve(ns);
    if (e == cudaSuccess) e = h->bend_map.reserve(nbd);
    if (e == cudaSuccess && nb) e = cudaMemsetAsync(link_owner, 0x7f, sizeof(int) * nb, st);
    if (e == cudaSuccess && nb) e = cudaMemsetAsync(bend_owner, 0x7f, sizeof(int) * nb, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(totals, 0, 2 * sizeof(int), st);
    if (e != cudaSuccess) return cuda_status(e);
    if (nb && (ns || nbd))
        k_claim<<<grid_for(nmax), kThreads, 0, st>>>(pos, d_sb, ns, d_bb, nbd, link_owner, bend_owner);
    h->chain.n_pos = nb;
    if (nb) {
        // owners still at the fill hold no link / bend
        k_chain_fill<<<grid_for(nb), kThreads, 0, st>>>(nb, link_owner, bend_owner, d_sk, d_sl, d_bk, d_bt,
                                                        h->chain_flags.raw(), h->chain_link_p.raw(),
                                                        h->chain_bend_p.raw());
    }
    // leftovers: flags, ranks, totals
    int left[2] = {0, 0};
    if (ns || nbd) {
        k_left_flags<<<grid_for(nmax), kThreads, 0, st>>>(pos, d_sb, ns, d_bb, nbd, link_owner, bend_owner, ls, lb);
        auto scan = [&](const int* in, int n, int* out, int* sums, int* total) {
            if (n <= 0) return;
            const int blocks = (n + kScanBlock - 1) / kScanBlock;
            k_scan_local<<<blocks, kScanBlock, 0, st>>>(in, n, out, sums);
            k_scan_block_sums<<<1, 32, 0, st>>>(sums, blocks, total);
            k_scan_apply<<<grid_for(n), kThreads, 0, st>>>(out, n, sums);
        };
        scan(ls, ns, ls_rank, sums_s, totals);
        scan(lb, nbd, lb_rank, sums_b, totals + 1);
        e = cudaMemcpyAsync(left, totals, sizeof left, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_status(e);
    }
    ff.n_stretch = left[0];
    ff.n_bend = left[1];
    e = h->stretch_bs.reserve(left[0]);
    if (e == cudaSuccess) e = h->stretch_p.reserve(left[0]);
    if (e == cudaSuccess) e = h->bend_bs.reserve(left[1]);
    if (e == cudaSuccess) e = h->bend_p.reserve(left[1]);
    if (e != cudaSuccess) return cuda_status(e);
    if (ns || nbd)
        k_left_write<<<grid_for(nmax), kThreads, 0, st>>>(pos, d_sb, d_sk, d_sl, ns, ls, ls_rank, d_bb, d_bk, d_bt,
                                                          nbd, lb, lb_rank, h->stretch_bs.raw(), h->stretch_p.raw(),
                                                          h->bend_bs.raw(), h->bend_p.raw(), h->stretch_map.raw(),
                                                          h->bend_map.raw());
    h->n_stretch_in = ns;
    h->n_bend_in = nbd;

    // generic records
    ff.n_linker = nl;
    ff.n_motor = nm;
    ff.n_branch = nr;
    ff.branch_mask = nr ? (s->branch_ff_mask & 0xF) : 0;
    ff.n_excl = ne;
    ff.n_boundary = nbo;
    ff.n_planes = np;
    e = h->linker_bs.reserve(nl);
    if (e == cudaSuccess) e = h->linker_p.reserve(nl);
    if (e == cudaSuccess) e = h->motor_bs.reserve(nm);
    if (e == cudaSuccess) e = h->motor_p.reserve(nm);
    if (e == cudaSuccess) e = h->branch_bs.reserve(nr);
    if (e == cudaSuccess) e = h->branch_pa.reserve(nr);
    if (e == cudaSuccess) e = h->branch_pb.reserve(nr);
    if (e == cudaSuccess) e = h->excl_bs.reserve(ne);
    if (e == cudaSuccess) e = h->excl_krs.reserve(ne);
    if (e == cudaSuccess) e = h->boundary_bs.reserve(nbo);
    if (e == cudaSuccess) e = h->boundary_p.reserve(nbo);
    if (e == cudaSuccess) e = h->boundary_plane.reserve(nbo);
    if (e == cudaSuccess) e = h->planes.reserve(np);
    if (e != cudaSuccess) return cuda_status(e);
    if (nl)
        k_springs<<<grid_for(nl), kThreads, 0, st>>>(pos, d_lb, d_lk, d_ll, d_l1, d_l2, nl, h->linker_bs.raw(),
                                                     h->linker_p.raw());
    if (nm)
        k_springs<<<grid_for(nm), kThreads, 0, st>>>(pos, d_mb, d_mk, d_ml, d_m1, d_m2, nm, h->motor_bs.raw(),
                                                     h->motor_p.raw());
    if (nr)
        k_branches<<<grid_for(nr), kThreads, 0, st>>>(pos, d_rb, d_rp, d_rsk, d_rsl, d_rbk, d_rbt, d_rdk, d_rpk, nr,
                                                      h->branch_bs.raw(), h->branch_pa.raw(), h->branch_pb.raw());
    if (ne) k_excl<<<grid_for(ne), kThreads, 0, st>>>(pos, d_eb, d_ek, d_el, ne, h->excl_bs.raw(), h->excl_krs.raw());
    if (nbo || np)
        k_boundary<<<grid_for(nbo > np ? nbo : np), kThreads, 0, st>>>(pos, d_ob, d_ok, d_os, nbo, d_pn, np, d_pe,
                                                                       h->boundary_bs.raw(), h->boundary_p.raw(),
                                                                       h->boundary_plane.raw(), h->planes.raw());
    e = cudaGetLastError();
    // the caller's arrays may be released on return
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e);
    return refresh_device_ff(h);
}

}  // namespace mb
