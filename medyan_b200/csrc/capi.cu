// capi.cu — the C ABI declared in include/medyan_b200.h: handle lifetime,
// host-side validation and packing of the vectorized force fields, and the
// energy/force entry points. The minimizer and the neighbor list are in
// cg.cu and nl.cu.
#include <cstdio>
#include <cstring>
#include <vector>

#include "handle.h"

using namespace mb;

namespace mb {

namespace {
thread_local cudaError_t t_last_cuda_error = cudaSuccess;
}

medyan_status cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return MEDYAN_OK;
    t_last_cuda_error = e;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return MEDYAN_ERR_NO_DEVICE;
    return MEDYAN_ERR_CUDA;
}

namespace {

bool check_offsets(const int32_t* bs, long long n, int32_t n_beads) {
    const long long lim = 3LL * n_beads;
    for (long long i = 0; i < n; ++i) {
        const int32_t v = bs[i];
        if (v < 0 || v >= lim || v % 3 != 0) return false;
    }
    return true;
}

template <class T>
const T* nz(const T* p, long long n) { return n > 0 ? p : nullptr; }

}  // namespace

// Validates every array of a vectorization (sizes, null pointers, bead
// offsets) before anything touches the device.
medyan_status validate_system(const medyan_system* s) {
    if (!s || s->n_beads < 0) return MEDYAN_ERR_INVALID_ARG;
    if (s->n_stretch < 0 || s->n_bend < 0 || s->n_linker < 0 || s->n_motor < 0 || s->n_branch < 0 ||
        s->n_excl < 0 || s->n_boundary < 0 || s->n_planes < 0)
        return MEDYAN_ERR_INVALID_ARG;
    const int nb = s->n_beads;
    if (s->n_stretch && (!s->stretch_beads || !s->stretch_k || !s->stretch_l0)) return MEDYAN_ERR_INVALID_ARG;
    if (s->n_bend && (!s->bend_beads || !s->bend_k || !s->bend_theta0)) return MEDYAN_ERR_INVALID_ARG;
    if (s->n_linker && (!s->linker_beads || !s->linker_k || !s->linker_l0 || !s->linker_pos1 || !s->linker_pos2))
        return MEDYAN_ERR_INVALID_ARG;
    if (s->n_motor && (!s->motor_beads || !s->motor_k || !s->motor_l0 || !s->motor_pos1 || !s->motor_pos2))
        return MEDYAN_ERR_INVALID_ARG;
    if (s->n_branch) {
        if (!s->branch_beads || !s->branch_pos) return MEDYAN_ERR_INVALID_ARG;
        const int m = s->branch_ff_mask;
        if ((m & 1) && (!s->branch_stretch_k || !s->branch_stretch_l0)) return MEDYAN_ERR_INVALID_ARG;
        if ((m & 2) && (!s->branch_bend_k || !s->branch_bend_theta0)) return MEDYAN_ERR_INVALID_ARG;
        if ((m & 4) && !s->branch_dihedral_k) return MEDYAN_ERR_INVALID_ARG;
        if ((m & 8) && !s->branch_position_k) return MEDYAN_ERR_INVALID_ARG;
    }
    if (s->n_excl && (!s->excl_beads || !s->excl_k || !s->excl_eqlen)) return MEDYAN_ERR_INVALID_ARG;
    if (s->n_boundary) {
        if (!s->boundary_beads || !s->boundary_k || !s->boundary_slen || !s->plane_eq || !s->plane_nneighbors ||
            s->n_planes <= 0)
            return MEDYAN_ERR_INVALID_ARG;
        long long tot = 0;
        for (int p = 0; p < s->n_planes; ++p) {
            if (s->plane_nneighbors[p] < 0) return MEDYAN_ERR_INVALID_ARG;
            tot += s->plane_nneighbors[p];
        }
        if (tot != s->n_boundary) return MEDYAN_ERR_INVALID_ARG;
    }
    if (!check_offsets(s->stretch_beads, 2LL * s->n_stretch, nb)) return MEDYAN_ERR_INDEX_RANGE;
    if (!check_offsets(s->bend_beads, 3LL * s->n_bend, nb)) return MEDYAN_ERR_INDEX_RANGE;
    if (!check_offsets(s->linker_beads, 4LL * s->n_linker, nb)) return MEDYAN_ERR_INDEX_RANGE;
    if (!check_offsets(s->motor_beads, 4LL * s->n_motor, nb)) return MEDYAN_ERR_INDEX_RANGE;
    if (!check_offsets(s->branch_beads, 4LL * s->n_branch, nb)) return MEDYAN_ERR_INDEX_RANGE;
    if (!check_offsets(s->excl_beads, 4LL * s->n_excl, nb)) return MEDYAN_ERR_INDEX_RANGE;
    if (!check_offsets(s->boundary_beads, (long long)s->n_boundary, nb)) return MEDYAN_ERR_INDEX_RANGE;
    return MEDYAN_OK;
}

// Packs the vectorization into the device records of DeviceFF with host
// loops: the same records as upload_system_device (vectorize.cu), which
// create and update use; kept as the reference for it
// (medyan_mech_set_host_packing).
medyan_status upload_system(medyan_mech* h, const medyan_system* s) {
    cudaStream_t st = h->stream;
    std::vector<int2> i2;
    std::vector<int4> i4;
    std::vector<double2> d2;
    std::vector<double4> d4, d4b;
    std::vector<double> d1;
    std::vector<int> ii, pl;
    DeviceFF& ff = h->ff;
    const int bonded_block = ff.bonded_block, excl_block = ff.excl_block;  // launch shapes survive an update
    ff = DeviceFF{};
    ff.bonded_block = bonded_block;
    ff.excl_block = excl_block;
    ff.n_beads = s->n_beads;
    cudaError_t e = cudaSuccess;
#define UPLOAD(buf, vec)                                                              \
    do {                                                                              \
        e = (buf).assign(vec.data(), vec.size(), st);                                 \
        if (e != cudaSuccess) return cuda_status(e);                                  \
    } while (0)

    // the internal bead order is fixed by the first vectorization
    if ((int)h->order_host.size() != s->n_beads) {
        chain_order(s, h->order_host);
        h->pos_host.assign(s->n_beads, 0);
        h->identity_order = true;
        for (int p = 0; p < s->n_beads; ++p) {
            h->pos_host[h->order_host[p]] = p;
            if (h->order_host[p] != p) h->identity_order = false;
        }
        if (!h->identity_order) UPLOAD(h->order, h->order_host);
        e = h->stage.reserve(3 * (size_t)s->n_beads);
        if (e != cudaSuccess) return cuda_status(e);
    }
    const std::vector<int>& pos = h->pos_host;
    auto R = [&](int32_t off) { return 3 * pos[off / 3]; };  // external offset -> internal offset

    // filament chains take every stretching link and bend that fits; the rest
    // stays on the generic path
    ChainHost chs;
    build_chains(s, pos, chs);
    UPLOAD(h->chain_flags, chs.flags);
    UPLOAD(h->chain_link_p, chs.link_p);
    UPLOAD(h->chain_bend_p, chs.bend_p);
    h->chain.n_pos = s->n_beads;

    // caller's interaction -> chain position or leftover record
    {
        std::vector<int> sm(s->n_stretch), bm(s->n_bend);
        for (int i = 0; i < s->n_stretch; ++i) sm[i] = pos[s->stretch_beads[2 * i] / 3];
        for (int q = 0; q < (int)chs.left_stretch.size(); ++q) sm[chs.left_stretch[q]] = -1 - q;
        for (int i = 0; i < s->n_bend; ++i) bm[i] = pos[s->bend_beads[3 * i + 1] / 3];
        for (int q = 0; q < (int)chs.left_bend.size(); ++q) bm[chs.left_bend[q]] = -1 - q;
        UPLOAD(h->stretch_map, sm);
        UPLOAD(h->bend_map, bm);
        h->n_stretch_in = s->n_stretch;
        h->n_bend_in = s->n_bend;
    }

    ff.n_stretch = (int)chs.left_stretch.size();
    i2.resize(ff.n_stretch);
    d2.resize(ff.n_stretch);
    for (int q = 0; q < ff.n_stretch; ++q) {
        const int i = chs.left_stretch[q];
        i2[q] = make_int2(R(s->stretch_beads[2 * i]), R(s->stretch_beads[2 * i + 1]));
        d2[q] = make_double2(s->stretch_k[i], s->stretch_l0[i]);
    }
    UPLOAD(h->stretch_bs, i2);
    UPLOAD(h->stretch_p, d2);

    ff.n_bend = (int)chs.left_bend.size();
    i4.resize(ff.n_bend);
    d2.resize(ff.n_bend);
    for (int q = 0; q < ff.n_bend; ++q) {
        const int i = chs.left_bend[q];
        i4[q] = make_int4(R(s->bend_beads[3 * i]), R(s->bend_beads[3 * i + 1]), R(s->bend_beads[3 * i + 2]), 0);
        d2[q] = make_double2(s->bend_k[i], s->bend_theta0[i]);
    }
    UPLOAD(h->bend_bs, i4);
    UPLOAD(h->bend_p, d2);

    auto pack_spring = [&](int n, const int32_t* bs, const double* k, const double* l0, const double* p1,
                           const double* p2) {
        i4.resize(n);
        d4.resize(n);
        for (int i = 0; i < n; ++i) {
            i4[i] = make_int4(R(bs[4 * i]), R(bs[4 * i + 1]), R(bs[4 * i + 2]), R(bs[4 * i + 3]));
            d4[i] = make_double4(k[i], l0[i], p1[i], p2[i]);
        }
    };
    ff.n_linker = s->n_linker;
    pack_spring(s->n_linker, s->linker_beads, s->linker_k, s->linker_l0, s->linker_pos1, s->linker_pos2);
    UPLOAD(h->linker_bs, i4);
    UPLOAD(h->linker_p, d4);
    ff.n_motor = s->n_motor;
    pack_spring(s->n_motor, s->motor_beads, s->motor_k, s->motor_l0, s->motor_pos1, s->motor_pos2);
    UPLOAD(h->motor_bs, i4);
    UPLOAD(h->motor_p, d4);

    ff.n_branch = s->n_branch;
    ff.branch_mask = s->n_branch ? (s->branch_ff_mask & 0xF) : 0;
    i4.resize(s->n_branch);
    d4.resize(s->n_branch);
    d4b.resize(s->n_branch);
    auto at = [](const double* p, int i) { return p ? p[i] : 0.0; };
    for (int i = 0; i < s->n_branch; ++i) {
        const int32_t* b = s->branch_beads + 4 * i;
        i4[i] = make_int4(R(b[0]), R(b[1]), R(b[2]), R(b[3]));
        d4[i] = make_double4(s->branch_pos[i], at(s->branch_stretch_k, i), at(s->branch_stretch_l0, i),
                             at(s->branch_bend_k, i));
        d4b[i] = make_double4(at(s->branch_bend_theta0, i), at(s->branch_dihedral_k, i),
                              at(s->branch_position_k, i), 0.0);
    }
    UPLOAD(h->branch_bs, i4);
    UPLOAD(h->branch_pa, d4);
    UPLOAD(h->branch_pb, d4b);

    ff.n_excl = s->n_excl;
    i4.resize(s->n_excl);
    d1.resize(s->n_excl);
    for (int i = 0; i < s->n_excl; ++i) {
        const int32_t* b = s->excl_beads + 4 * i;
        i4[i] = make_int4(R(b[0]), R(b[1]), R(b[2]), R(b[3]));
        // kRepScaled = krep * eqLength_1 * eqLength_2, CylinderExclVolRepulsion.cpp:355
        d1[i] = s->excl_k[i] * s->excl_eqlen[2 * i] * s->excl_eqlen[2 * i + 1];
    }
    UPLOAD(h->excl_bs, i4);
    UPLOAD(h->excl_krs, d1);

    ff.n_boundary = s->n_boundary;
    ff.n_planes = s->n_planes;
    ii.resize(s->n_boundary);
    for (int i = 0; i < s->n_boundary; ++i) ii[i] = R(s->boundary_beads[i]);
    d2.resize(s->n_boundary);
    pl.resize(s->n_boundary);
    {
        int t = 0;
        for (int p = 0; p < s->n_planes; ++p)
            for (int c = 0; c < s->plane_nneighbors[p]; ++c, ++t) pl[t] = p;
    }
    for (int i = 0; i < s->n_boundary; ++i) d2[i] = make_double2(s->boundary_k[i], s->boundary_slen[i]);
    d4.resize(s->n_planes);
    for (int p = 0; p < s->n_planes; ++p)
        d4[p] = make_double4(s->plane_eq[4 * p], s->plane_eq[4 * p + 1], s->plane_eq[4 * p + 2], s->plane_eq[4 * p + 3]);
    UPLOAD(h->boundary_bs, ii);
    UPLOAD(h->boundary_p, d2);
    UPLOAD(h->boundary_plane, pl);
    UPLOAD(h->planes, d4);
#undef UPLOAD
    return refresh_device_ff(h);
}

// Re-derives DeviceFF pointers and the block table from the owned buffers,
// and sizes the energy scratch.
medyan_status refresh_device_ff(medyan_mech* h) {
    DeviceFF& ff = h->ff;
    ff.stretch_bs = h->stretch_bs.ptr();
    ff.stretch_p = h->stretch_p.ptr();
    ff.bend_bs = h->bend_bs.ptr();
    ff.bend_p = h->bend_p.ptr();
    ff.linker_bs = h->linker_bs.ptr();
    ff.linker_p = h->linker_p.ptr();
    ff.motor_bs = h->motor_bs.ptr();
    ff.motor_p = h->motor_p.ptr();
    ff.branch_bs = h->branch_bs.ptr();
    ff.branch_pa = h->branch_pa.ptr();
    ff.branch_pb = h->branch_pb.ptr();
    ff.excl_bs = h->excl_bs.ptr();
    ff.excl_krs = h->excl_krs.ptr();
    ff.boundary_bs = h->boundary_bs.ptr();
    ff.boundary_p = h->boundary_p.ptr();
    ff.boundary_plane = h->boundary_plane.ptr();
    ff.planes = h->planes.ptr();
    h->chain.flags = h->chain_flags.raw();
    h->chain.link_p = h->chain_link_p.raw();
    h->chain.bend_p = h->chain_bend_p.raw();
    const int counts[6] = {ff.n_stretch, ff.n_bend, ff.n_linker, ff.n_motor, ff.n_branch, ff.n_boundary};
    ff.seg[0] = 0;
    const int bb = bonded_block_of(ff);
    for (int q = 0; q < 6; ++q) ff.seg[q + 1] = ff.seg[q] + (counts[q] + bb - 1) / bb;
    h->es.n_blocks_chain = h->chain.n_pos > 0 ? chain_blocks(h->chain) : 0;
    h->es.n_blocks_bonded = ff.seg[6];
    h->es.n_blocks_excl = excl_blocks(ff);
    const size_t need = (size_t)kMaxLambda * (h->es.total() + 1) * 4;
    cudaError_t e = h->partial.reserve(need);
    {
        // fused-pass scratch; the group tickets start at zero (stream-ordered
        // after every pass already enqueued on the handle's stream)
        // (sized for both fused layouts, so a change of layout needs no reallocation)
        const PassGeometry pg = pass_geometry(h->chain, ff, false), ps = pass_geometry(h->chain, ff, true);
        const int rows = pg.rows > ps.rows ? pg.rows : ps.rows;
        const int groups = pg.groups > ps.groups ? pg.groups : ps.groups;
        if (e == cudaSuccess) e = h->pass_rows.reserve((size_t)rows * MEDYAN_FF_COUNT);
        if (e == cudaSuccess) e = h->pass_group_rows.reserve((size_t)groups * MEDYAN_FF_COUNT);
        if (e == cudaSuccess) e = h->pass_group_ticket.reserve((size_t)groups);
        if (e == cudaSuccess) e = h->pass_fgroup_ticket.reserve((size_t)groups);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(h->pass_group_ticket.raw(), 0, sizeof(unsigned int) * h->pass_group_ticket.cap,
                                h->stream);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(h->pass_fgroup_ticket.raw(), 0, sizeof(unsigned int) * h->pass_fgroup_ticket.cap,
                                h->stream);
    }
    {
        // fallback queues with room for every pair (energies: every pair at
        // every step size of a pass), so a pair the analytic formulas reject
        // always gets its quadrature, as in the reference, however many
        // there are
        const size_t n_ex = ff.n_excl > 0 ? (size_t)ff.n_excl : 0;
        const size_t ecap = n_ex * kMaxLambda > (size_t)kFallbackCap ? n_ex * kMaxLambda : (size_t)kFallbackCap;
        const size_t fcap = n_ex > (size_t)kFallbackCap ? n_ex : (size_t)kFallbackCap;
        if (e == cudaSuccess) e = h->e_fb_list.reserve(ecap);
        if (e == cudaSuccess) e = h->f_fb_list.reserve(fcap);
        h->es.fb_list = h->e_fb_list.raw();
        h->fs.fb_list = h->f_fb_list.raw();
        h->es.fb_cap = (int)h->e_fb_list.cap;
        h->fs.fb_cap = (int)h->f_fb_list.cap;
    }
    if (e != cudaSuccess) return cuda_status(e);
    h->es.partial = h->partial.ptr();
    h->ff_gen++;
    return MEDYAN_OK;
}

medyan_status sync_status(medyan_mech* h) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_status(e);
    return MEDYAN_OK;
}

// Energy at x (+ lam*d when d is set) for the lambda set in device memory;
// results land in h->es.out.
void enqueue_energy(medyan_mech* h, const double* x, const double* d, const LambdaSet* lam, cudaStream_t s) {
    launch_energy(h->chain, h->ff, h->prec, x, d, lam, h->es, s, &h->fork);
}

void enqueue_forces(medyan_mech* h, const double* x, double* f, cudaStream_t s) {
    enqueue_force_target(h, x, ForceTarget{f, nullptr, nullptr, nullptr, nullptr, nullptr, h->deterministic, h->fs.status},
                         h->fs, s);
}

void enqueue_force_target(medyan_mech* h, const double* x, const ForceTarget& t, const ForceScratch& fs,
                          cudaStream_t s) {
    if (h->pass_layout == 0 || h->pass_layout == 2)
        launch_pass_fused(h->chain, h->ff, h->prec, x, &t, false, nullptr, h->es, fs, h->pass_scratch(),
                          h->pass_scratch_forces(), s, &h->fork, h->pass_layout == 2);
    else
        launch_forces(h->chain, h->ff, h->prec, x, t, fs, s, &h->fork);
}

cudaError_t coords_to_device(medyan_mech* h, const double* host, double* dev, cudaStream_t s) {
    const int n3 = 3 * h->n_beads;
    if (n3 == 0) return cudaSuccess;
    if (h->identity_order) return cudaMemcpyAsync(dev, host, sizeof(double) * n3, cudaMemcpyHostToDevice, s);
    cudaError_t e = cudaMemcpyAsync(h->stage.raw(), host, sizeof(double) * n3, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) launch_to_internal(n3, h->order.raw(), h->stage.raw(), dev, s);
    return e == cudaSuccess ? cudaGetLastError() : e;
}

cudaError_t coords_to_host(medyan_mech* h, const double* dev, double* host, cudaStream_t s) {
    const int n3 = 3 * h->n_beads;
    if (n3 == 0) return cudaSuccess;
    if (h->identity_order) return cudaMemcpyAsync(host, dev, sizeof(double) * n3, cudaMemcpyDeviceToHost, s);
    launch_to_external(n3, h->order.raw(), dev, h->stage.raw(), s);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, h->stage.raw(), sizeof(double) * n3, cudaMemcpyDeviceToHost, s);
    return e;
}

static cudaError_t count_kernel_nodes(cudaGraph_t g, int* out) {
    size_t n = 0;
    cudaError_t e = cudaGraphGetNodes(g, nullptr, &n);
    if (e != cudaSuccess) return e;
    std::vector<cudaGraphNode_t> nodes(n);
    if (n) e = cudaGraphGetNodes(g, nodes.data(), &n);
    int k = 0;
    for (size_t i = 0; i < n && e == cudaSuccess; ++i) {
        cudaGraphNodeType t;
        e = cudaGraphNodeGetType(nodes[i], &t);
        if (e == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
    }
    *out = k;
    return e;
}

// Captures and instantiates pass `which` when the force fields changed.
cudaError_t ensure_pass_graph(medyan_mech* h, int which) {
    if (h->pass_graph[which] && h->pass_graph_gen[which] == h->ff_gen) return cudaSuccess;
    if (h->pass_graph[which]) cudaGraphExecDestroy(h->pass_graph[which]);
    h->pass_graph[which] = nullptr;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    const ForceTarget t{h->f.raw(), nullptr, nullptr, nullptr, nullptr, nullptr, h->deterministic, h->fs.status};
    if (h->pass_layout == 0 || h->pass_layout == 2)
        launch_pass_fused(h->chain, h->ff, h->prec, h->x.raw(), which == kPassEnergy ? nullptr : &t,
                          which != kPassForces, h->lam_zero.raw(), h->es, h->fs, h->pass_scratch(),
                          h->pass_scratch_forces(), h->stream, &h->fork, h->pass_layout == 2);
    else if (which == kPassBoth)
        launch_evaluate(h->chain, h->ff, h->prec, h->x.raw(), nullptr, h->lam_zero.raw(), t, h->es, h->fs, h->stream,
                        &h->fork);
    else if (which == kPassEnergy)
        enqueue_energy(h, h->x.raw(), nullptr, h->lam_zero.raw(), h->stream);
    else
        enqueue_forces(h, h->x.raw(), h->f.raw(), h->stream);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(h->stream, &g);
    if (e == cudaSuccess) e = count_kernel_nodes(g, &h->pass_kernels[which]);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&h->pass_graph[which], g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        h->pass_graph[which] = nullptr;
        return e;
    }
    h->pass_graph_gen[which] = h->ff_gen;
    return cudaSuccess;
}

cudaError_t launch_pass(medyan_mech* h, int which) {
    cudaError_t e = ensure_pass_graph(h, which);
    if (e != cudaSuccess) return e;
    return cudaGraphLaunch(h->pass_graph[which], h->stream);
}

}  // namespace mb

medyan_status medyan_mech::init() {
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    for (int k = 0; k < kForkWays && e == cudaSuccess; ++k)
        e = cudaStreamCreateWithFlags(&fork.side[k], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork.fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork.mid, cudaEventDisableTiming);
    for (int k = 0; k < kForkWays && e == cudaSuccess; ++k)
        e = cudaEventCreateWithFlags(&fork.join[k], cudaEventDisableTiming);
    if (e == cudaSuccess) e = init_excl_kernels();
    if (e == cudaSuccess) e = init_pass_kernels();
    const size_t n3 = 3 * (size_t)n_beads;
    if (e == cudaSuccess) e = x.reserve(n3);
    if (e == cudaSuccess) e = f.reserve(n3);
    if (e == cudaSuccess) e = energy_out.reserve((size_t)kMaxLambda * (MEDYAN_FF_COUNT + 1));
    if (e == cudaSuccess) e = e_fb_count.reserve(1);
    if (e == cudaSuccess) e = e_bad.reserve(kMaxLambda);
    if (e == cudaSuccess) e = e_fb_list.reserve(kFallbackCap);
    if (e == cudaSuccess) e = e_stage.reserve((size_t)kMaxLambda * kFinishBlocks * MEDYAN_FF_COUNT);
    if (e == cudaSuccess) e = e_ticket.reserve(1);
    if (e == cudaSuccess) e = f_fb_count.reserve(1);
    if (e == cudaSuccess) e = f_fb_list.reserve(kFallbackCap);
    if (e == cudaSuccess) e = force_status.reserve(1);
    if (e == cudaSuccess) e = lam_zero.reserve(1);
    if (e == cudaSuccess) e = pass_ticket.reserve(2);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&small), sizeof(*small));
    if (e != cudaSuccess) return cuda_status(e);
    cudaMemsetAsync(x.raw(), 0, sizeof(double) * (n3 ? n3 : 1), stream);
    cudaMemsetAsync(e_fb_count.raw(), 0, sizeof(int), stream);
    cudaMemsetAsync(e_bad.raw(), 0, sizeof(int) * kMaxLambda, stream);
    cudaMemsetAsync(e_ticket.raw(), 0, sizeof(unsigned int), stream);
    cudaMemsetAsync(f_fb_count.raw(), 0, sizeof(int), stream);
    cudaMemsetAsync(force_status.raw(), 0, sizeof(int), stream);
    cudaMemsetAsync(pass_ticket.raw(), 0, 2 * sizeof(unsigned int), stream);
    LambdaSet z{};
    z.K = 1;
    e = lam_zero.assign(&z, 1, stream);
    if (e != cudaSuccess) return cuda_status(e);
    es.fb_count = e_fb_count.raw();
    es.fb_list = e_fb_list.raw();
    es.bad = e_bad.raw();
    es.out = energy_out.raw();
    es.stage = e_stage.raw();
    es.ticket = e_ticket.raw();
    fs.fb_count = f_fb_count.raw();
    fs.fb_list = f_fb_list.raw();
    fs.status = force_status.raw();
    return cuda_status(cudaStreamSynchronize(stream));
}

medyan_mech::~medyan_mech() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (cg_graph) cudaGraphExecDestroy(cg_graph);
    if (cg_pinned) cudaFreeHost(cg_pinned);
    if (small) cudaFreeHost(small);
    for (auto& g : pass_graph)
        if (g) cudaGraphExecDestroy(g);
    destroy_async(this);
    destroy_nl(this);
    for (auto& sd : fork.side)
        if (sd) cudaStreamDestroy(sd);
    if (fork.fork) cudaEventDestroy(fork.fork);
    if (fork.mid) cudaEventDestroy(fork.mid);
    for (auto& ev : fork.join)
        if (ev) cudaEventDestroy(ev);
    if (stream) cudaStreamDestroy(stream);
}

// ---------------------------------------------------------------------------
extern "C" {

int32_t medyan_abi_version(void) { return 2; }

const char* medyan_last_cuda_error(void) {
    return t_last_cuda_error == cudaSuccess ? "" : cudaGetErrorName(t_last_cuda_error);
}

const char* medyan_status_string(int32_t s) {
    switch (s) {
        case MEDYAN_OK: return "ok";
        case MEDYAN_ERR_INVALID_ARG: return "invalid argument";
        case MEDYAN_ERR_INDEX_RANGE: return "bead index out of range";
        case MEDYAN_ERR_NONFINITE: return "non-finite energy or force";
        case MEDYAN_ERR_ITER_CAP: return "iteration cap reached";
        case MEDYAN_ERR_CUDA: return "CUDA error";
        case MEDYAN_ERR_OUT_OF_GRID: return "cylinder outside the neighbor-list grid";
        case MEDYAN_ERR_LINE_SEARCH: return "line search failed";
        case MEDYAN_ERR_NO_DEVICE: return "no CUDA device";
        case MEDYAN_ERR_CAPACITY: return "output buffer too small";
        case MEDYAN_ERR_UNSUPPORTED: return "unsupported option";
        default: return "unknown status";
    }
}

medyan_status medyan_mech_create(const medyan_system* sys, int32_t precision, medyan_mech** out) {
    if (!out) return MEDYAN_ERR_INVALID_ARG;
    *out = nullptr;
    if (precision != MEDYAN_PREC_FP64 && precision != MEDYAN_PREC_MIXED) return MEDYAN_ERR_INVALID_ARG;
    medyan_status v = validate_system(sys);
    if (v != MEDYAN_OK) return v;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e);
    auto* h = new medyan_mech();
    h->device = dev;
    h->prec = precision;
    h->n_beads = sys->n_beads;
    medyan_status st = h->init();
    if (st == MEDYAN_OK) st = upload_system_device(h, sys);
    if (st == MEDYAN_OK) st = sync_status(h);
    if (st != MEDYAN_OK) {
        delete h;
        return st;
    }
    *out = h;
    return MEDYAN_OK;
}

medyan_status medyan_mech_update(medyan_mech* h, const medyan_system* sys) {
    if (!h || !sys || sys->n_beads != h->n_beads) return MEDYAN_ERR_INVALID_ARG;
    medyan_status v = validate_system(sys);
    if (v != MEDYAN_OK) return v;
    medyan_status st = h->host_packing ? upload_system(h, sys) : upload_system_device(h, sys);
    if (st != MEDYAN_OK) return st;
    return sync_status(h);
}

medyan_status medyan_mech_set_host_packing(medyan_mech* h, int32_t on) {
    if (!h || (on != 0 && on != 1)) return MEDYAN_ERR_INVALID_ARG;
    h->host_packing = on;
    return MEDYAN_OK;
}

medyan_status medyan_mech_destroy(medyan_mech* h) {
    if (!h) return MEDYAN_ERR_INVALID_ARG;
    delete h;
    return MEDYAN_OK;
}

medyan_status medyan_mech_set_coords(medyan_mech* h, const double* coord) {
    if (!h || (!coord && h->n_beads)) return MEDYAN_ERR_INVALID_ARG;
    cudaError_t e = coords_to_device(h, coord, h->x.raw(), h->stream);
    if (e != cudaSuccess) return cuda_status(e);
    return sync_status(h);
}

medyan_status medyan_mech_get_coords(medyan_mech* h, double* coord) {
    if (!h || (!coord && h->n_beads)) return MEDYAN_ERR_INVALID_ARG;
    cudaError_t e = coords_to_host(h, h->x.raw(), coord, h->stream);
    if (e != cudaSuccess) return cuda_status(e);
    return sync_status(h);
}

medyan_status medyan_mech_energy(medyan_mech* h, double* e_total, double* e_per_ff) {
    if (!h || !e_total) return MEDYAN_ERR_INVALID_ARG;
    cudaError_t e = launch_pass(h, kPassEnergy);
    if (e != cudaSuccess) return cuda_status(e);
    double* out = h->small->energy;
    e = cudaMemcpyAsync(out, h->energy_out.ptr(), sizeof h->small->energy, cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess) return cuda_status(e);
    medyan_status st = sync_status(h);
    if (st != MEDYAN_OK) return st;
    *e_total = out[MEDYAN_FF_COUNT];
    if (e_per_ff) std::memcpy(e_per_ff, out, sizeof(double) * MEDYAN_FF_COUNT);
    if (std::isinf(out[MEDYAN_FF_COUNT])) return MEDYAN_ERR_NONFINITE;
    return MEDYAN_OK;
}

medyan_status medyan_mech_forces(medyan_mech* h, double* force_out) {
    if (!h || (!force_out && h->n_beads)) return MEDYAN_ERR_INVALID_ARG;
    cudaError_t e = launch_pass(h, kPassForces);
    if (e != cudaSuccess) return cuda_status(e);
    e = coords_to_host(h, h->f.raw(), force_out, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&h->small->force_status, h->force_status.ptr(), sizeof(int), cudaMemcpyDeviceToHost,
                            h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->force_status.ptr(), 0, sizeof(int), h->stream);
    if (e != cudaSuccess) return cuda_status(e);
    medyan_status st = sync_status(h);
    if (st != MEDYAN_OK) return st;
    return h->small->force_status ? MEDYAN_ERR_NONFINITE : MEDYAN_OK;
}

medyan_status medyan_mech_enqueue_energy(medyan_mech* h) {
    if (!h) return MEDYAN_ERR_INVALID_ARG;
    return cuda_status(launch_pass(h, kPassEnergy));
}

medyan_status medyan_mech_enqueue_forces(medyan_mech* h) {
    if (!h) return MEDYAN_ERR_INVALID_ARG;
    return cuda_status(launch_pass(h, kPassForces));
}

medyan_status medyan_mech_enqueue_evaluate(medyan_mech* h) {
    if (!h) return MEDYAN_ERR_INVALID_ARG;
    return cuda_status(launch_pass(h, kPassBoth));
}

medyan_status medyan_mech_set_deterministic(medyan_mech* h, int32_t on) {
    if (!h || (on != 0 && on != 1)) return MEDYAN_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);  // no pass may still write the old way
    if (e != cudaSuccess) return cuda_status(e);
    if (h->deterministic != on) {
        h->deterministic = on;
        h->ff_gen++;  // recapture the passes and the minimizer's graph
    }
    return MEDYAN_OK;
}

medyan_status medyan_mech_synchronize(medyan_mech* h) {
    if (!h) return MEDYAN_ERR_INVALID_ARG;
    int status = 0;
    cudaError_t e = cudaMemcpyAsync(&status, h->force_status.ptr(), sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->force_status.ptr(), 0, sizeof(int), h->stream);
    if (e != cudaSuccess) return cuda_status(e);
    medyan_status st = sync_status(h);
    if (st != MEDYAN_OK) return st;
    return status ? MEDYAN_ERR_NONFINITE : MEDYAN_OK;
}

void* medyan_mech_stream(medyan_mech* h) { return h ? (void*)h->stream : nullptr; }

int32_t medyan_mech_pass_kernel_count(medyan_mech* h, int32_t which) {
    if (!h || which < 0 || which > 2) return -1;
    if (cudaSetDevice(h->device) != cudaSuccess) return -1;
    if (ensure_pass_graph(h, which) != cudaSuccess) return -1;
    return h->pass_kernels[which];
}

medyan_status medyan_mech_device_buffers(medyan_mech* h, double** coord, double** force, double** energy) {
    if (!h) return MEDYAN_ERR_INVALID_ARG;
    if (coord) *coord = h->x.raw();
    if (force) *force = h->f.raw();
    if (energy) *energy = h->energy_out.raw();
    return MEDYAN_OK;
}

medyan_status medyan_mech_evaluate(medyan_mech* h, const double* coord, double* e_total, double* e_per_ff,
                                   double* force_out) {
    if (!h || !coord || !e_total || !force_out) return MEDYAN_ERR_INVALID_ARG;
    cudaError_t e = coords_to_device(h, coord, h->x.raw(), h->stream);
    if (e != cudaSuccess) return cuda_status(e);
    e = launch_pass(h, kPassBoth);
    if (e != cudaSuccess) return cuda_status(e);
    double* out = h->small->energy;
    e = cudaMemcpyAsync(out, h->energy_out.ptr(), sizeof h->small->energy, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = coords_to_host(h, h->f.raw(), force_out, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&h->small->force_status, h->force_status.ptr(), sizeof(int), cudaMemcpyDeviceToHost,
                            h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->force_status.ptr(), 0, sizeof(int), h->stream);
    if (e != cudaSuccess) return cuda_status(e);
    medyan_status st = sync_status(h);
    if (st != MEDYAN_OK) return st;
    *e_total = out[MEDYAN_FF_COUNT];
    if (e_per_ff) std::memcpy(e_per_ff, out, sizeof(double) * MEDYAN_FF_COUNT);
    if (h->small->force_status) return MEDYAN_ERR_NONFINITE;
    if (std::isinf(out[MEDYAN_FF_COUNT])) return MEDYAN_ERR_NONFINITE;
    return MEDYAN_OK;
}

}  // extern "C"
