// chain.cu — filament stretching and bending as one bead-centric pass.
//
// At upload the stretching links (b1 -> b2) and bending triplets
// (b1, b2, b3) are arranged into chains: every bead gets one chain position,
// beads of a filament consecutive, links between consecutive positions and
// each bend centred on its middle bead (FilamentStretching::vectorize,
// Filament/FilamentStretching.cpp:24-44, FilamentBending::vectorize,
// Filament/FilamentBending.cpp:28-66, produce exactly this structure).
// Interactions that do not fit (a bead with two outgoing links, a bend whose
// beads are not consecutive on a chain, links closing a cycle) stay on the
// generic per-interaction path.
//
// The force kernel stages a tile of chain positions (+2 on each side) in
// shared memory, evaluates each link and each bend once, and writes each
// bead's force with a plain store: no atomics, no index loads beyond one
// offset per bead, and every bead (including beads on no chain) is written,
// so the pass also initializes the force array for the potentials that add
// atomically afterwards. The energy kernel evaluates the link and bend owned
// by each position at up to kMaxLambda step sizes from one read of x and d.
#include <algorithm>
#include <vector>

#include "handle.h"
#include "potentials.cuh"

namespace mb {

namespace {

constexpr int kTile = 256;
constexpr unsigned char kLink = 1, kBend = 2;

template <class R>
struct ChainSmem {
    double cx[kTile + 4], cy[kTile + 4], cz[kTile + 4];  // positions p0-2 .. p0+T+1
    R fs[kTile + 1][3];                                  // link (q, q+1) force on q+1, q = p0-1 .. p0+T-1
    R fr1[kTile + 2][3], fr2[kTile + 2][3];              // bend centred at q = p0-1 .. p0+T
    unsigned char fl[kTile + 2];                         // flags of q = p0-1 .. p0+T
};

template <class R>
__global__ void __launch_bounds__(kTile) k_chain_forces(const ChainDev ch, const double* __restrict__ x,
                                                       const ForceTarget tgt) {
    if (tgt.skip && *tgt.skip) return;
    __shared__ ChainSmem<R> S;
    double* __restrict__ f = target_force(tgt);
    const double* __restrict__ d = tgt.d;
    const double lam = tgt.lam ? *tgt.lam : 0.0;
    const int n = ch.n_pos;
    for (int p0 = blockIdx.x * kTile; p0 < n; p0 += gridDim.x * kTile) {
        // stage positions p0-2 .. p0+T+1 and flags p0-1 .. p0+T
        for (int t = threadIdx.x; t < kTile + 4; t += kTile) {
            const int q = p0 - 2 + t;
            double X = 0, Y = 0, Z = 0;
            if (q >= 0 && q < n) {
                const int o = ch.bead[q];
                X = x[o];
                Y = x[o + 1];
                Z = x[o + 2];
                if (d) {
                    X = move1(X, lam, d[o]);
                    Y = move1(Y, lam, d[o + 1]);
                    Z = move1(Z, lam, d[o + 2]);
                }
            }
            S.cx[t] = X;
            S.cy[t] = Y;
            S.cz[t] = Z;
        }
        for (int t = threadIdx.x; t < kTile + 2; t += kTile) {
            const int q = p0 - 1 + t;
            S.fl[t] = (q >= 0 && q < n) ? ch.flags[q] : 0;
        }
        __syncthreads();
        // terms of centres q = p0-1+t for t in [0, T+2)
        for (int t = threadIdx.x; t < kTile + 2; t += kTile) {
            const int q = p0 - 1 + t;
            const unsigned char fl = S.fl[t];
            const int c = t + 1;  // index of position q in the coordinate tile
            if (t < kTile + 1) {
                T3<R> F{0, 0, 0};
                if (fl & kLink) {
                    double2 lp = ch.link_p[q];
                    F = stretch_force<R>(V3{S.cx[c], S.cy[c], S.cz[c]}, V3{S.cx[c + 1], S.cy[c + 1], S.cz[c + 1]},
                                         lp.x, lp.y);
                }
                S.fs[t][0] = F.x;
                S.fs[t][1] = F.y;
                S.fs[t][2] = F.z;
            }
            T3<R> A{0, 0, 0}, B{0, 0, 0};
            if (fl & kBend) {
                double2 bp = ch.bend_p[q];
                V3 c0{S.cx[c - 1], S.cy[c - 1], S.cz[c - 1]}, c1{S.cx[c], S.cy[c], S.cz[c]},
                    c2{S.cx[c + 1], S.cy[c + 1], S.cz[c + 1]};
                bend_force<R>(diff<R>(c0, c1), diff<R>(c1, c2), bp.x, bp.y, A, B);
            }
            S.fr1[t][0] = A.x;
            S.fr1[t][1] = A.y;
            S.fr1[t][2] = A.z;
            S.fr2[t][0] = B.x;
            S.fr2[t][1] = B.y;
            S.fr2[t][2] = B.z;
        }
        __syncthreads();
        const int p = p0 + threadIdx.x;
        if (p < n) {
            const int t = threadIdx.x + 1;  // centre p in the term arrays
            double out[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                // link (p-1, p) acts on p; link (p, p+1) reacts on p;
                // bends centred at p-1 (third bead), p (middle), p+1 (first bead);
                // summed in double
                out[k] = double(S.fs[t - 1][k]) - double(S.fs[t][k]) + double(S.fr2[t - 1][k]) +
                         (double(S.fr1[t][k]) - double(S.fr2[t][k])) - double(S.fr1[t + 1][k]);
            }
            const int o = ch.bead[p];
            f[o] = out[0];
            f[o + 1] = out[1];
            f[o + 2] = out[2];
        }
        __syncthreads();
    }
}

template <class R>
__global__ void __launch_bounds__(kTile) k_chain_energy(const ChainDev ch, const double* __restrict__ x,
                                                       const double* __restrict__ d,
                                                       const LambdaSet* __restrict__ lset,
                                                       double* __restrict__ partial, int nblk_total, int blk_off) {
    __shared__ double sm[4 * 32];
    __shared__ double cx[2][kTile + 2], cy[2][kTile + 2], cz[2][kTile + 2];  // x and d, positions p0-1 .. p0+T
    const int n = ch.n_pos;
    const int K = lset ? lset->K : 1;
    double acc[kMaxLambda][2];
#pragma unroll
    for (int k = 0; k < kMaxLambda; ++k) acc[k][0] = acc[k][1] = 0.0;
    for (int p0 = blockIdx.x * kTile; p0 < n; p0 += gridDim.x * kTile) {
        for (int t = threadIdx.x; t < kTile + 2; t += kTile) {
            const int q = p0 - 1 + t;
            double X = 0, Y = 0, Z = 0, DX = 0, DY = 0, DZ = 0;
            if (q >= 0 && q < n) {
                const int o = ch.bead[q];
                X = x[o];
                Y = x[o + 1];
                Z = x[o + 2];
                if (d) {
                    DX = d[o];
                    DY = d[o + 1];
                    DZ = d[o + 2];
                }
            }
            cx[0][t] = X; cy[0][t] = Y; cz[0][t] = Z;
            cx[1][t] = DX; cy[1][t] = DY; cz[1][t] = DZ;
        }
        __syncthreads();
        const int p = p0 + threadIdx.x;
        if (p < n) {
            const unsigned char fl = ch.flags[p];
            const int c = threadIdx.x + 1;
            double2 lp = {0, 0}, bp = {0, 0};
            if (fl & kLink) lp = ch.link_p[p];
            if (fl & kBend) bp = ch.bend_p[p];
            if (fl) {
                for (int k = 0; k < K; ++k) {
                    const double lam = lset ? lset->lam[k] : 0.0;
                    auto P = [&](int i) {
                        V3 v{cx[0][i], cy[0][i], cz[0][i]};
                        return d ? move3(v, lam, V3{cx[1][i], cy[1][i], cz[1][i]}) : v;
                    };
                    const V3 pc = P(c), pn = P(c + 1);
                    if (fl & kLink) acc[k][0] += stretch_energy<R>(pc, pn, lp.x, lp.y);
                    if (fl & kBend) acc[k][1] += bend_energy<R>(diff<R>(P(c - 1), pc), diff<R>(pc, pn), bp.x, bp.y);
                }
            }
        }
        __syncthreads();
    }
    for (int k = 0; k < K; ++k) {
        double e[2] = {acc[k][0], acc[k][1]};
        block_sum<2>(e, sm);
        if (threadIdx.x == 0) {
            double* o = partial + ((size_t)k * nblk_total + blk_off + blockIdx.x) * 4;
            o[0] = e[0];
            o[1] = e[1];
            o[2] = 0.0;
            o[3] = 0.0;
        }
    }
}

}  // namespace

int chain_blocks(const ChainDev& ch) {
    int tiles = (ch.n_pos + kTile - 1) / kTile;
    int cap = 148 * 4;
    return tiles < cap ? (tiles < 1 ? 1 : tiles) : cap;
}

void launch_chain_forces(const ChainDev& ch, int prec, const double* x, const ForceTarget& t, cudaStream_t s) {
    if (ch.n_pos <= 0) return;
    const int g = (ch.n_pos + kTile - 1) / kTile;
    if (prec == MEDYAN_PREC_MIXED)
        k_chain_forces<float><<<g, kTile, 0, s>>>(ch, x, t);
    else
        k_chain_forces<double><<<g, kTile, 0, s>>>(ch, x, t);
}

void launch_chain_energy(const ChainDev& ch, int prec, const double* x, const double* d, const LambdaSet* lam,
                         double* partial, int nblk_total, int blk_off, cudaStream_t s) {
    if (ch.n_pos <= 0) return;
    const int g = chain_blocks(ch);
    if (prec == MEDYAN_PREC_MIXED)
        k_chain_energy<float><<<g, kTile, 0, s>>>(ch, x, d, lam, partial, nblk_total, blk_off);
    else
        k_chain_energy<double><<<g, kTile, 0, s>>>(ch, x, d, lam, partial, nblk_total, blk_off);
}

// Host: arrange stretching links and bends into chains. Returns the leftover
// (non-chain) stretching and bending interaction indices.
void build_chains(const medyan_system* s, ChainHost& out) {
    const int nb = s->n_beads;
    std::vector<int> next(nb, -1), prev(nb, -1), link_id(nb, -1);
    out.left_stretch.clear();
    out.left_bend.clear();
    for (int i = 0; i < s->n_stretch; ++i) {
        const int a = s->stretch_beads[2 * i] / 3, c = s->stretch_beads[2 * i + 1] / 3;
        if (a != c && next[a] < 0 && prev[c] < 0) {
            next[a] = c;
            prev[c] = a;
            link_id[a] = i;
        } else {
            out.left_stretch.push_back(i);
        }
    }
    // break cycles: walk from every bead without a predecessor; beads left
    // unvisited lie on cycles, whose link into the smallest bead is dropped
    std::vector<int> pos(nb, -1);
    std::vector<int> order;
    order.reserve(nb);
    auto walk = [&](int h) {
        for (int b = h; b >= 0 && pos[b] < 0; b = next[b]) {
            pos[b] = (int)order.size();
            order.push_back(b);
        }
    };
    for (int b = 0; b < nb; ++b)
        if (prev[b] < 0) walk(b);
    for (int b = 0; b < nb; ++b) {
        if (pos[b] >= 0) continue;
        // b is on an unvisited cycle; cut the link entering b
        const int a = prev[b];
        out.left_stretch.push_back(link_id[a]);
        next[a] = -1;
        link_id[a] = -1;
        prev[b] = -1;
        walk(b);
    }
    std::sort(out.left_stretch.begin(), out.left_stretch.end());
    const int n = (int)order.size();
    out.bead.assign(n, 0);
    out.flags.assign(n, 0);
    out.link_p.assign(n, make_double2(0, 0));
    out.bend_p.assign(n, make_double2(0, 0));
    for (int p = 0; p < n; ++p) {
        const int b = order[p];
        out.bead[p] = 3 * b;
        if (next[b] >= 0) {
            out.flags[p] |= kLink;
            const int i = link_id[b];
            out.link_p[p] = make_double2(s->stretch_k[i], s->stretch_l0[i]);
        }
    }
    for (int i = 0; i < s->n_bend; ++i) {
        const int b1 = s->bend_beads[3 * i] / 3, b2 = s->bend_beads[3 * i + 1] / 3, b3 = s->bend_beads[3 * i + 2] / 3;
        const int p = pos[b2];
        if (next[b1] == b2 && next[b2] == b3 && !(out.flags[p] & kBend)) {
            out.flags[p] |= kBend;
            out.bend_p[p] = make_double2(s->bend_k[i], s->bend_theta0[i]);
        } else {
            out.left_bend.push_back(i);
        }
    }
}

}  // namespace mb
