// Persistent level kernels of the device-driven loop, precision fp32
// (cp_graph_kernels.cuh), by family and block-size variant.
#include "cp_graph_kernels.cuh"

using namespace cpb;

namespace {
template <int FAM>
void* pick(int v) {
    switch (v) {
    case 0: return (void*)k_level_persist<FAM, 1, 64>;
    case 1: return (void*)k_level_persist<FAM, 1, 128>;
    case 2: return (void*)k_level_persist<FAM, 1, 256>;
    case 3: return (void*)k_level_persist<FAM, 1, 512>;
    default: return (void*)k_level_persist<FAM, 1, 1024>;
    }
}
}  // namespace

void* cp_graph_kernel_fp32(int fam, int variant) {
    switch (fam) {
    case 0: return pick<0>(variant);
    case 1: return pick<1>(variant);
    case 2: return pick<2>(variant);
    case 3: return pick<3>(variant);
    case 4: return pick<4>(variant);
    default: return pick<5>(variant);
    }
}

void* cp_graph_kernel_net_fp32(int fam) {
    switch (fam) {
    case 0: return (void*)k_level_persist_net<0, 1>;
    case 1: return (void*)k_level_persist_net<1, 1>;
    case 2: return (void*)k_level_persist_net<2, 1>;
    case 3: return (void*)k_level_persist_net<3, 1>;
    case 4: return (void*)k_level_persist_net<4, 1>;
    default: return (void*)k_level_persist_net<5, 1>;
    }
}
