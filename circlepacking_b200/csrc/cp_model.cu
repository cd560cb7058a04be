// Learned proposal model (criterion order and split axis per box).
#include "cp_common.h"
#include "cp_engine.h"
#include "cp_worklist.cuh"

cp_status cp_model_hints(cp_prover* p, int fam, const cpb::BoxList& in, size_t begin, size_t count, uint8_t** axis,
                         uint8_t** order) {
    (void)p, (void)fam, (void)in, (void)begin, (void)count, (void)axis, (void)order;
    return CP_ERR_INVALID;  // no model loaded
}

void cp_model_free(cp_prover* p) { (void)p; }
