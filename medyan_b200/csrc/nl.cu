// nl.cu — cylinder neighbor list on the device (placeholder until the
// cell-list kernels land).
#include "handle.h"

struct medyan_mech::NL {};

namespace mb {
void destroy_nl(medyan_mech* h) {
    delete h->nl;
    h->nl = nullptr;
}
}  // namespace mb

extern "C" {
medyan_status medyan_nl_build(const medyan_cylinders*, const double*, int32_t, const medyan_nl_params*, int32_t*,
                              int64_t, int64_t*) {
    return MEDYAN_ERR_UNSUPPORTED;
}
medyan_status medyan_mech_set_cylinders(medyan_mech*, const medyan_cylinders*, const medyan_nl_params*,
                                        const medyan_boundary_params*) {
    return MEDYAN_ERR_UNSUPPORTED;
}
medyan_status medyan_mech_rebuild_neighbors(medyan_mech*, int64_t*, int64_t*) { return MEDYAN_ERR_UNSUPPORTED; }
medyan_status medyan_mech_get_excl_volume(medyan_mech*, int32_t*, double*, double*, int64_t, int64_t*) {
    return MEDYAN_ERR_UNSUPPORTED;
}
}
