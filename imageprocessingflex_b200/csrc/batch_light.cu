// batch_light.cu -- the light-class persistent batch kernel (median k >= 7),
// the separable group launches with K <= 13, and the separable tile geometry
// table.
#include "batch_kernel.cuh"

namespace ipfc {

cudaError_t batch_launch_light(const BatchItem* items, const BatchTile* tiles, int ntiles, unsigned* counter, int grid,
                               size_t smem, cudaStream_t s) {
    return batch_launch_class<0>(items, tiles, ntiles, counter, grid, smem, s);
}

cudaError_t batch_occupancy_light(size_t smem, int* occ) { return batch_occupancy_class<0>(smem, occ); }

// Separable group launches with K <= 13 taps.
bool batch_sep_group_light(int k, int c, const SepGroup& g, int n, int max_tiles, cudaStream_t s, cudaError_t* e) {
    return batch_sep_group_case<3>(k, c, g, n, max_tiles, s, e) || batch_sep_group_case<5>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<7>(k, c, g, n, max_tiles, s, e) || batch_sep_group_case<9>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<11>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<13>(k, c, g, n, max_tiles, s, e);
}

namespace {

template <int K, int C>
struct SepGeomU8 {
    using G = FastGeom<K, C, 4>;
};

template <int K>
bool sep_geom_lookup(int k, int C, int* px, size_t* smem) {
    if (k != K) return false;
    if (C == 1) {
        *px = SepGeomU8<K, 1>::G::PX;
        *smem = SepGeomU8<K, 1>::G::SMEM;
    } else if (C == 3) {
        *px = SepGeomU8<K, 3>::G::PX;
        *smem = SepGeomU8<K, 3>::G::SMEM;
    } else {
        *px = SepGeomU8<K, 4>::G::PX;
        *smem = SepGeomU8<K, 4>::G::SMEM;
    }
    return true;
}

bool sep_geom(int K, int C, int* px, size_t* smem) {
    return sep_geom_lookup<3>(K, C, px, smem) || sep_geom_lookup<5>(K, C, px, smem) ||
           sep_geom_lookup<7>(K, C, px, smem) || sep_geom_lookup<9>(K, C, px, smem) ||
           sep_geom_lookup<11>(K, C, px, smem) || sep_geom_lookup<13>(K, C, px, smem) ||
           sep_geom_lookup<15>(K, C, px, smem) || sep_geom_lookup<17>(K, C, px, smem) ||
           sep_geom_lookup<19>(K, C, px, smem) || sep_geom_lookup<21>(K, C, px, smem) ||
           sep_geom_lookup<23>(K, C, px, smem) || sep_geom_lookup<25>(K, C, px, smem);
}

}  // namespace

int batch_sep_px(int K, int C) {
    int px = 0;
    size_t smem = 0;
    return sep_geom(K, C, &px, &smem) ? px : 0;
}

size_t batch_sep_smem(int K, int C) {
    int px = 0;
    size_t smem = 0;
    return sep_geom(K, C, &px, &smem) ? smem : 0;
}

}  // namespace ipfc
