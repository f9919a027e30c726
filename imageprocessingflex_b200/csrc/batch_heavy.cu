// batch_heavy.cu -- the separable group launches with 15 to 25 taps.  The
// heavy class holds only group launches: no queue tile belongs to it.
#include "batch_kernel.cuh"

namespace ipfc {

// Separable group launches with 15 to 25 taps.
bool batch_sep_group_heavy(int k, int c, const SepGroup& g, int n, int max_tiles, cudaStream_t s, cudaError_t* e) {
    return batch_sep_group_case<15>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<17>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<19>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<21>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<23>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<25>(k, c, g, n, max_tiles, s, e);
}

}  // namespace ipfc
