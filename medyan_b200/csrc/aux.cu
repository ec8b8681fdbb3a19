// aux.cu — force magnitudes for the chemistry after a minimization.
//
// ForceFieldManager::assignallforcemags (src/Mechanics/ForceField/ForceFieldManager.cpp:346-351)
// hands each force field's per-interaction "stretchforce" array to the
// chemistry: the linker and motor tension k (L - l0) (LinkerStretchingHarmonic.cpp:227-293,
// MotorGhostStretchingHarmonic.cpp:274-339) and, per branch point, the force
// each branching force field puts on the third bead of its bead set
// (BranchingStretchingHarmonic.cpp:235-275, BranchingBendingCosine.cpp:330-359,
// BranchingDihedralCosine.cpp:500-505, BranchingPositionCosine.cpp:437-447),
// added in force-field order. One FP64 kernel over the records at the
// handle's coordinates, built with --fmad=false so the tension of a spring
// at its rest length comes out as exactly zero, as in the reference.
#include <algorithm>

#include "handle.h"
#include "potentials.cuh"

namespace mb {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double tension(const V3& c1, const V3& c2, const V3& c3, const V3& c4, double4 p) {
    const V3 v1 = midpoint(c1, c2, p.z), v2 = midpoint(c3, c4, p.w);
    const double dx = v2.x - v1.x, dy = v2.y - v1.y, dz = v2.z - v1.z;
    const double dist = sqrt(dx * dx + dy * dy + dz * dz);
    const double invL = 1 / dist;
    const double f0 = p.x * (dist - p.y) * invL;
    return f0 / invL;
}

__global__ void __launch_bounds__(kThreads) k_force_mags(const DeviceFF ff, const double* __restrict__ x,
                                                         double* __restrict__ lin, double* __restrict__ mot,
                                                         double* __restrict__ br) {
    const int n = ff.n_linker + ff.n_motor + ff.n_branch;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        if (t < ff.n_linker + ff.n_motor) {
            const bool L = t < ff.n_linker;
            const int i = L ? t : t - ff.n_linker;
            double* out = L ? lin : mot;
            if (!out) continue;
            const int4 q = L ? ff.linker_bs[i] : ff.motor_bs[i];
            const double4 p = L ? ff.linker_p[i] : ff.motor_p[i];
            out[i] = tension(load3(x + q.x), load3(x + q.y), load3(x + q.z), load3(x + q.w), p);
            continue;
        }
        if (!br) continue;
        const int i = t - ff.n_linker - ff.n_motor;
        const int4 q = ff.branch_bs[i];
        const double4 pa = ff.branch_pa[i], pb = ff.branch_pb[i];
        const V3 c1 = load3(x + q.x), c2 = load3(x + q.y), c3 = load3(x + q.z), c4 = load3(x + q.w);
        double fx = 0.0, fy = 0.0, fz = 0.0;
        if (ff.branch_mask & 1) {  // -f0 r1 on the third bead
            const T3<double> g = branch_stretch_force<double>(c1, c2, c3, pa.y, pa.z, pa.x);
            fx += -g.x;
            fy += -g.y;
            fz += -g.z;
        }
        if (ff.branch_mask & 2) {
            T3<double> Fr1, Fr2;
            bend_force<double>(diff<double>(c1, c2), diff<double>(c3, c4), pa.w, pb.x, Fr1, Fr2);
            fx += -Fr2.x;
            fy += -Fr2.y;
            fz += -Fr2.z;
        }
        if (ff.branch_mask & 4) {
            T3<double> L1, L2, L3, L4;
            branch_dihedral_force<double>(c1, c2, c3, c4, pb.y, pa.x, L1, L2, L3, L4);
            fx += L3.x;
            fy += L3.y;
            fz += L3.z;
        }
        if (ff.branch_mask & 8) {
            T3<double> P1, P2, P3;
            branch_position_force<double>(c1, c2, c3, pb.z, pa.x, P1, P2, P3);
            fx += P3.x;
            fy += P3.y;
            fz += P3.z;
        }
        br[3 * i] = fx;
        br[3 * i + 1] = fy;
        br[3 * i + 2] = fz;
    }
}

}  // namespace

}  // namespace mb

using namespace mb;

extern "C" medyan_status medyan_mech_force_magnitudes(medyan_mech* h, double* linker_stretch, double* motor_stretch,
                                                      double* branch_force) {
    if (!h) return MEDYAN_ERR_INVALID_ARG;
    const DeviceFF& ff = h->ff;
    const int n = ff.n_linker + ff.n_motor + ff.n_branch;
    if (n == 0) return MEDYAN_OK;
    cudaError_t e = cudaSetDevice(h->device);
    cudaStream_t s = h->stream;
    DevBuf<double> out;
    const size_t nl = ff.n_linker, nm = ff.n_motor, nb = 3 * (size_t)ff.n_branch;
    if (e == cudaSuccess) e = out.reserve(nl + nm + nb);
    if (e != cudaSuccess) return cuda_status(e);
    double* d = out.raw();
    const int g = std::min(148 * 8, (n + kThreads - 1) / kThreads);
    k_force_mags<<<g, kThreads, 0, s>>>(ff, h->x.raw(), linker_stretch ? d : nullptr,
                                        motor_stretch ? d + nl : nullptr, branch_force ? d + nl + nm : nullptr);
    e = cudaGetLastError();
    if (e == cudaSuccess && linker_stretch && nl)
        e = cudaMemcpyAsync(linker_stretch, d, sizeof(double) * nl, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && motor_stretch && nm)
        e = cudaMemcpyAsync(motor_stretch, d + nl, sizeof(double) * nm, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && branch_force && nb)
        e = cudaMemcpyAsync(branch_force, d + nl + nm, sizeof(double) * nb, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e);
}
