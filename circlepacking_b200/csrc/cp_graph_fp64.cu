// Persistent level kernels of the device-driven loop, precision fp64
// (cp_graph_kernels.cuh), by family and block-size variant.
#include "cp_graph_kernels.cuh"

using namespace cpb;

namespace {
template <int FAM>
void* pick(int v) {
    switch (v) {
    case 0: return (void*)k_level_persist<FAM, 0, 64>;
    case 1: return (void*)k_level_persist<FAM, 0, 128>;
    case 2: return (void*)k_level_persist<FAM, 0, 256>;
    case 3: return (void*)k_level_persist<FAM, 0, 512>;
    default: return (void*)k_level_persist<FAM, 0, 1024>;
    }
}
}  // namespace

void* cp_graph_kernel_fp64(int fam, int variant) {
    switch (fam) {
    case 0: return pick<0>(variant);
    case 1: return pick<1>(variant);
    case 2: return pick<2>(variant);
    case 3: return pick<3>(variant);
    case 4: return pick<4>(variant);
    default: return pick<5>(variant);
    }
}

void* cp_graph_kernel_net_fp64(int fam) {
    switch (fam) {
    case 0: return (void*)k_level_persist_net<0, 0>;
    case 1: return (void*)k_level_persist_net<1, 0>;
    case 2: return (void*)k_level_persist_net<2, 0>;
    case 3: return (void*)k_level_persist_net<3, 0>;
    case 4: return (void*)k_level_persist_net<4, 0>;
    default: return (void*)k_level_persist_net<5, 0>;
    }
}
