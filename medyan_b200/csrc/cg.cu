// cg.cu — device-resident conjugate-gradient minimizer (placeholder).
#include "handle.h"

extern "C" {
medyan_status medyan_cg_minimize(medyan_mech*, const medyan_cg_params*, double*, double*, medyan_min_result*) {
    return MEDYAN_ERR_UNSUPPORTED;
}
}
