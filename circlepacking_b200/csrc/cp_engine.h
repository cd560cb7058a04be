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
// Trace recording (cp_model_collect): labels a sample of the chunk's boxes
// before the engine evaluates it; a no-op unless a collection is running.
bool cp_model_collecting(cp_prover* p);
cp_status cp_model_collect_chunk(cp_prover* p, int fam, const cpb::BoxList& in, size_t begin, size_t count,
                                 const double* tab_t, const double* tab_v, int tab_n, double tab_h);

// Persistent level kernels of the graph engine (cp_graph_fp64.cu / cp_graph_fp32.cu).
void* cp_graph_kernel_fp64(int fam, int variant);
void* cp_graph_kernel_fp32(int fam, int variant);
// Persistent level kernels that run the proposal network inline (128 threads).
void* cp_graph_kernel_net_fp64(int fam);
void* cp_graph_kernel_net_fp32(int fam);
// The trained network of a family for kernels that run it inline: BF16 views,
// FP32 master parameters and the completion-wait limit (CP_ERR_INVALID when
// the family has no model).
cp_status cp_model_net_params(cp_prover* p, int fam, const void** views, const float** master, int* wait_limit);

// Pieces of the refinement engine reused by the static-scratch entry point
// (cp_noalloc.cu).  Counters: cp_engine_counter_words() 64-bit words.
size_t cp_engine_counter_words();
cp_status cp_engine_launch_table(double lambda_lo, double h, int n, double* t, double* v, cudaStream_t st);
cp_status cp_engine_launch_level(int fam, int prec, int variant, const cpb::BoxList& in, size_t begin, size_t count,
                                 const cpb::BoxList* out, unsigned long long out_base, unsigned long long* counters,
                                 const double* tab_t, const double* tab_v, int tab_n, double tab_h, int policy,
                                 int max_depth, cudaStream_t st);
// Reads the overflow flag and children count of a counter block copied to the host.
bool cp_engine_overflowed(const unsigned long long* h_counters);
unsigned long long cp_engine_children(const unsigned long long* h_counters);
void cp_engine_fill_report(const unsigned long long* h_counters, cp_refine_report* r);
