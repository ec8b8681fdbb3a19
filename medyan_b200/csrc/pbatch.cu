// pbatch.cu — packing a batch of replica handles into one set of arrays
// (see pbatch.h). Packing is a device-to-device gather from the replicas'
// own arrays (their internal bead order, their device-built neighbor lists),
// with bead offsets shifted by each replica's base and every replica's
// records padded to whole blocks.
#include <vector>

#include "pbatch.h"

namespace mb {

namespace {

constexpr int kPackThreads = 256;

// dst[i] = src[i] + shift for i < n_src; padding: pad in the first component
// of each record, 0 in the others.
__global__ void k_pack_index(const int* __restrict__ src, int n_src, int n_dst, int shift, int pad, int comps,
                             int* __restrict__ dst) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_dst; i += gridDim.x * blockDim.x)
        dst[i] = i < n_src ? src[i] + shift : ((i % comps) == 0 ? pad : 0);
}

int pad_to(int n, int b) { return (n + b - 1) / b * b; }

cudaError_t pack_index(const void* src, int n_rec, int n_pad, int comps, int shift, int pad, void* dst,
                       cudaStream_t s) {
    const int nd = n_pad * comps;
    if (nd == 0) return cudaSuccess;
    int g = (nd + kPackThreads - 1) / kPackThreads;
    if (g > 1024) g = 1024;
    k_pack_index<<<g, kPackThreads, 0, s>>>(static_cast<const int*>(src), n_rec * comps, nd, shift, pad, comps,
                                             static_cast<int*>(dst));
    return cudaGetLastError();
}

template <class T>
cudaError_t copy_rec(const T* src, int n, T* dst, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, sizeof(T) * n, cudaMemcpyDeviceToDevice, s);
}

}  // namespace

PackedBatch::~PackedBatch() {
    if (stream) cudaStreamSynchronize(stream);
    if (graph) cudaGraphExecDestroy(graph);
    for (auto& sd : fork.side)
        if (sd) cudaStreamDestroy(sd);
    if (fork.fork) cudaEventDestroy(fork.fork);
    for (auto& ev : fork.join)
        if (ev) cudaEventDestroy(ev);
    if (stream) cudaStreamDestroy(stream);
}

medyan_status pack_batch(PackedBatch& pb, const std::vector<medyan_mech*>& h) {
    const int R = (int)h.size();
    long long gen = 0;
    for (auto* r : h) gen += r->ff_gen;
    if (!pb.repack && pb.R == R && pb.gen == gen && (int)pb.base.size() == R + 1) return MEDYAN_OK;
    cudaError_t e = cudaSuccess;
    if (!pb.stream) {
        e = cudaStreamCreateWithFlags(&pb.stream, cudaStreamNonBlocking);
        for (int k = 0; k < kForkWays && e == cudaSuccess; ++k)
            e = cudaStreamCreateWithFlags(&pb.fork.side[k], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pb.fork.fork, cudaEventDisableTiming);
        for (int k = 0; k < kForkWays && e == cudaSuccess; ++k)
            e = cudaEventCreateWithFlags(&pb.fork.join[k], cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_status(e);
    }
    for (auto* r : h) {
        e = cudaStreamSynchronize(r->stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    cudaStream_t s = pb.stream;
    pb.R = R;
    pb.base.assign(R + 1, 0);
    // one branching mask for the batch
    int mask = -1;
    for (auto* r : h) {
        if (r->ff.n_branch == 0) continue;
        if (mask < 0) mask = r->ff.branch_mask;
        else if (mask != r->ff.branch_mask) return MEDYAN_ERR_UNSUPPORTED;
    }
    // per-replica padded counts and offsets
    enum { S_STRETCH, S_BEND, S_LINKER, S_MOTOR, S_BRANCH, S_BOUNDARY, S_EXCL, S_N };
    std::vector<int> cnt[S_N], off[S_N];
    int tot[S_N] = {0};
    std::vector<int> plane_base(R + 1, 0);
    for (int k = 0; k < S_N; ++k) {
        cnt[k].resize(R);
        off[k].resize(R + 1, 0);
    }
    for (int r = 0; r < R; ++r) {
        const DeviceFF& f = h[r]->ff;
        pb.base[r + 1] = pb.base[r] + h[r]->n_beads;
        plane_base[r + 1] = plane_base[r] + f.n_planes;
        const int n[S_N] = {f.n_stretch, f.n_bend, f.n_linker, f.n_motor, f.n_branch, f.n_boundary, f.n_excl};
        for (int k = 0; k < S_N; ++k) {
            cnt[k][r] = n[k];
            off[k][r + 1] = off[k][r] + pad_to(n[k], k == S_EXCL ? pb.excl_block : pb.bonded_block);
        }
    }
    for (int k = 0; k < S_N; ++k) tot[k] = off[k][R];
    pb.nb = pb.base[R];
    const int nb = pb.nb;

    // buffers
    auto res = [&](auto& buf, size_t n) {
        if (e == cudaSuccess) e = buf.reserve(n ? n : 1);
    };
    res(pb.flags, nb);
    res(pb.link_p, nb);
    res(pb.bend_p, nb);
    res(pb.stretch_bs, tot[S_STRETCH]);
    res(pb.stretch_p, tot[S_STRETCH]);
    res(pb.bend_bs, tot[S_BEND]);
    res(pb.bend_pp, tot[S_BEND]);
    res(pb.linker_bs, tot[S_LINKER]);
    res(pb.linker_p, tot[S_LINKER]);
    res(pb.motor_bs, tot[S_MOTOR]);
    res(pb.motor_p, tot[S_MOTOR]);
    res(pb.branch_bs, tot[S_BRANCH]);
    res(pb.branch_pa, tot[S_BRANCH]);
    res(pb.branch_pb, tot[S_BRANCH]);
    res(pb.boundary_bs, tot[S_BOUNDARY]);
    res(pb.boundary_p, tot[S_BOUNDARY]);
    res(pb.boundary_plane, tot[S_BOUNDARY]);
    res(pb.excl_bs, tot[S_EXCL]);
    res(pb.excl_krs, tot[S_EXCL]);
    res(pb.planes, plane_base[R]);
    res(pb.x, 3 * (size_t)nb);
    if (e != cudaSuccess) return cuda_status(e);
    // parameters of padding records are zero
    auto zero = [&](auto& buf, size_t n, size_t sz) {
        if (e == cudaSuccess && n) e = cudaMemsetAsync(buf.raw(), 0, n * sz, s);
    };
    zero(pb.stretch_p, tot[S_STRETCH], sizeof(double2));
    zero(pb.bend_pp, tot[S_BEND], sizeof(double2));
    zero(pb.linker_p, tot[S_LINKER], sizeof(double4));
    zero(pb.motor_p, tot[S_MOTOR], sizeof(double4));
    zero(pb.branch_pa, tot[S_BRANCH], sizeof(double4));
    zero(pb.branch_pb, tot[S_BRANCH], sizeof(double4));
    zero(pb.boundary_p, tot[S_BOUNDARY], sizeof(double2));
    zero(pb.excl_krs, tot[S_EXCL], sizeof(double));

    for (int r = 0; r < R && e == cudaSuccess; ++r) {
        const medyan_mech* m = h[r];
        const DeviceFF& f = m->ff;
        const int b = pb.base[r], sh = 3 * b;
        const int nbr = m->n_beads;
        e = copy_rec(m->chain_flags.raw(), nbr, pb.flags.raw() + b, s);
        if (e == cudaSuccess) e = copy_rec(m->chain_link_p.raw(), nbr, pb.link_p.raw() + b, s);
        if (e == cudaSuccess) e = copy_rec(m->chain_bend_p.raw(), nbr, pb.bend_p.raw() + b, s);
        auto idx = [&](const void* src, int k, int comps, void* dst_base, int pad, int shift) {
            const int o = off[k][r];
            if (e == cudaSuccess)
                e = pack_index(src, cnt[k][r], off[k][r + 1] - o, comps, shift, pad,
                               static_cast<int*>(dst_base) + (size_t)o * comps, s);
        };
        idx(f.stretch_bs, S_STRETCH, 2, pb.stretch_bs.raw(), -1, sh);
        idx(f.bend_bs, S_BEND, 4, pb.bend_bs.raw(), -1, sh);
        idx(f.linker_bs, S_LINKER, 4, pb.linker_bs.raw(), -1, sh);
        idx(f.motor_bs, S_MOTOR, 4, pb.motor_bs.raw(), -1, sh);
        idx(f.branch_bs, S_BRANCH, 4, pb.branch_bs.raw(), -1, sh);
        idx(f.excl_bs, S_EXCL, 4, pb.excl_bs.raw(), -1, sh);
        idx(f.boundary_bs, S_BOUNDARY, 1, pb.boundary_bs.raw(), -1, sh);
        idx(f.boundary_plane, S_BOUNDARY, 1, pb.boundary_plane.raw(), 0, plane_base[r]);
        if (e == cudaSuccess) e = copy_rec(f.stretch_p, cnt[S_STRETCH][r], pb.stretch_p.raw() + off[S_STRETCH][r], s);
        if (e == cudaSuccess) e = copy_rec(f.bend_p, cnt[S_BEND][r], pb.bend_pp.raw() + off[S_BEND][r], s);
        if (e == cudaSuccess) e = copy_rec(f.linker_p, cnt[S_LINKER][r], pb.linker_p.raw() + off[S_LINKER][r], s);
        if (e == cudaSuccess) e = copy_rec(f.motor_p, cnt[S_MOTOR][r], pb.motor_p.raw() + off[S_MOTOR][r], s);
        if (e == cudaSuccess) e = copy_rec(f.branch_pa, cnt[S_BRANCH][r], pb.branch_pa.raw() + off[S_BRANCH][r], s);
        if (e == cudaSuccess) e = copy_rec(f.branch_pb, cnt[S_BRANCH][r], pb.branch_pb.raw() + off[S_BRANCH][r], s);
        if (e == cudaSuccess)
            e = copy_rec(f.boundary_p, cnt[S_BOUNDARY][r], pb.boundary_p.raw() + off[S_BOUNDARY][r], s);
        if (e == cudaSuccess) e = copy_rec(f.excl_krs, cnt[S_EXCL][r], pb.excl_krs.raw() + off[S_EXCL][r], s);
        if (e == cudaSuccess) e = copy_rec(f.planes, f.n_planes, pb.planes.raw() + plane_base[r], s);
    }
    if (e != cudaSuccess) return cuda_status(e);

    // the packed force-field view
    DeviceFF& ff = pb.ff;
    ff = DeviceFF{};
    ff.n_beads = nb;
    ff.n_stretch = tot[S_STRETCH];
    ff.n_bend = tot[S_BEND];
    ff.n_linker = tot[S_LINKER];
    ff.n_motor = tot[S_MOTOR];
    ff.n_branch = tot[S_BRANCH];
    ff.n_excl = tot[S_EXCL];
    ff.n_boundary = tot[S_BOUNDARY];
    ff.n_planes = plane_base[R];
    ff.branch_mask = mask < 0 ? 0 : mask;
    ff.stretch_bs = pb.stretch_bs.raw();
    ff.stretch_p = pb.stretch_p.raw();
    ff.bend_bs = pb.bend_bs.raw();
    ff.bend_p = pb.bend_pp.raw();
    ff.linker_bs = pb.linker_bs.raw();
    ff.linker_p = pb.linker_p.raw();
    ff.motor_bs = pb.motor_bs.raw();
    ff.motor_p = pb.motor_p.raw();
    ff.branch_bs = pb.branch_bs.raw();
    ff.branch_pa = pb.branch_pa.raw();
    ff.branch_pb = pb.branch_pb.raw();
    ff.excl_bs = pb.excl_bs.raw();
    ff.excl_krs = pb.excl_krs.raw();
    ff.boundary_bs = pb.boundary_bs.raw();
    ff.boundary_p = pb.boundary_p.raw();
    ff.boundary_plane = pb.boundary_plane.raw();
    ff.planes = pb.planes.raw();
    const int counts[6] = {ff.n_stretch, ff.n_bend, ff.n_linker, ff.n_motor, ff.n_branch, ff.n_boundary};
    ff.seg[0] = 0;
    const int B = pb.bonded_block, X = pb.excl_block, P = pb.chain_chunk;
    ff.bonded_block = B;
    ff.excl_block = X;
    for (int q = 0; q < 6; ++q) ff.seg[q + 1] = ff.seg[q] + (counts[q] + B - 1) / B;
    pb.ch = ChainDev{nb, pb.flags.raw(), pb.link_p.raw(), pb.bend_p.raw()};
    pb.ch.force_threads = pb.chain_threads;

    // chain energy chunks and per-replica row ranges
    std::vector<int4> table;
    std::vector<int> rows(9 * (R + 1), 0);
    int* rc = rows.data();
    int* rs = rows.data() + (R + 1);
    int* re = rows.data() + 7 * (R + 1);
    int* rp = rows.data() + 8 * (R + 1);
    const int seg_of[6] = {S_STRETCH, S_BEND, S_LINKER, S_MOTOR, S_BRANCH, S_BOUNDARY};
    for (int r = 0; r <= R; ++r) {
        rc[r] = (int)table.size();
        for (int q = 0; q < 6; ++q) rs[q * (R + 1) + r] = ff.seg[q] + off[seg_of[q]][r] / B;
        re[r] = off[S_EXCL][r] / X;
        rp[r] = off[S_EXCL][r];
        if (r == R) break;
        for (int p0 = pb.base[r]; p0 < pb.base[r + 1]; p0 += P)
            table.push_back(make_int4(r, p0, p0 + P < pb.base[r + 1] ? p0 + P : pb.base[r + 1], 0));
    }
    pb.n_chain_blocks = (int)table.size();
    // replica of every position, bonded block and excluded-volume block
    std::vector<int> rb(nb), rbb(ff.seg[6] > 0 ? ff.seg[6] : 1, 0), rbe(tot[S_EXCL] / X + 1, 0);
    for (int r = 0; r < R; ++r) {
        for (int p = pb.base[r]; p < pb.base[r + 1]; ++p) rb[p] = r;
        for (int q = 0; q < 6; ++q)
            for (int blk = rs[q * (R + 1) + r]; blk < rs[q * (R + 1) + r + 1]; ++blk) rbb[blk] = r;
        for (int blk = re[r]; blk < re[r + 1]; ++blk) rbe[blk] = r;
    }
    e = pb.chain_table.assign(table.data(), table.size(), s);
    if (e == cudaSuccess) e = pb.rep_bead.assign(rb.data(), rb.size(), s);
    if (e == cudaSuccess) e = pb.rep_bonded.assign(rbb.data(), rbb.size(), s);
    if (e == cudaSuccess) e = pb.rep_excl.assign(rbe.data(), rbe.size(), s);
    if (e == cudaSuccess) e = pb.act.reserve(R);
    if (e == cudaSuccess) {
        ff.act = pb.act.raw();
        ff.rep_bonded = pb.rep_bonded.raw();
        ff.rep_excl = pb.rep_excl.raw();
        pb.ch.rep = pb.rep_bead.raw();
        pb.ch.act = pb.act.raw();
    }
    if (e == cudaSuccess) e = pb.rows.assign(rows.data(), rows.size(), s);
    if (e == cudaSuccess) e = pb.base_dev.assign(pb.base.data(), pb.base.size(), s);

    // energy and force scratch
    EnergyScratch& es = pb.es;
    es.n_blocks_chain = pb.n_chain_blocks;
    es.n_blocks_bonded = ff.seg[6];
    es.n_blocks_excl = excl_blocks(ff);
    if (e == cudaSuccess) e = pb.partial.reserve((size_t)kMaxLambda * (es.total() + 1) * 4);
    if (e == cudaSuccess) e = pb.e_fb_count.reserve(1);
    if (e == cudaSuccess) e = pb.e_bad.reserve(kMaxLambda);
    if (e == cudaSuccess) e = pb.e_fb_list.reserve(kFallbackCap);
    if (e == cudaSuccess) e = pb.f_fb_count.reserve(1);
    if (e == cudaSuccess) e = pb.f_fb_list.reserve(kFallbackCap);
    if (e == cudaSuccess) e = pb.force_status.reserve(1);
    if (e == cudaSuccess) e = cudaMemsetAsync(pb.e_fb_count.raw(), 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(pb.e_bad.raw(), 0, sizeof(int) * kMaxLambda, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(pb.f_fb_count.raw(), 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(pb.force_status.raw(), 0, sizeof(int), s);
    if (e != cudaSuccess) return cuda_status(e);
    es.partial = pb.partial.raw();
    es.fb_count = pb.e_fb_count.raw();
    es.fb_list = pb.e_fb_list.raw();
    es.bad = pb.e_bad.raw();
    es.out = nullptr;  // batched results go to pb.out
    es.stage = nullptr;
    es.ticket = nullptr;
    pb.fs.fb_count = pb.f_fb_count.raw();
    pb.fs.fb_list = pb.f_fb_list.raw();
    pb.fs.status = pb.force_status.raw();
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    pb.gen = gen;
    pb.repack = false;
    return MEDYAN_OK;
}

}  // namespace mb
