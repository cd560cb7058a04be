// Internal interface between the engine and the learned model.
#pragma once
#include <cuda_runtime.h>

#include "cp_prover.h"

namespace cpb {
struct BoxList;
}

// The handle's stream, and the slot for the learned model's state.
cudaStream_t cp_prover_stream(cp_prover* p);
void*& cp_prover_model(cp_prover* p);

// Learned model hooks (cp_model.cu): per-box split axis / criterion order hints
// for boxes [begin, begin+count) of a worklist; device buffers owned by the model.
cp_status cp_model_hints(cp_prover* p, int fam, const cpb::BoxList& in, size_t begin, size_t count, uint8_t** axis,
                         uint8_t** order);
// Releases the model state of a handle.
void cp_model_free(cp_prover* p);
