// batch.cu -- host side of the batch API (ipfc_batch_*): items, the tile
// plan, the autotuner and the CUDA graph of a batch.
//
// Plan.  Every item is cut into the per-image kernels' tiles: separable
// items into strips of the kernel's strip width by chunks of R rows,
// median / morphology items into TX x TY tiles.  R and (TX, TY) come from
// the autotuner, keyed on (op, taps or ksize, channels, size class).  Items
// go to the light or heavy class (batch.cuh); within a class they are
// ordered by estimated cost per tile, most expensive first, and each item's
// tiles are consecutive, so the queue hands out the long tiles first and the
// short ones fill the tail (longest-processing-time order).
//
// Graph.  The first run of a plan captures, on two private streams: a
// memset of the two queue counters, then the heavy and the light persistent
// kernels as two parallel branches.  Later runs launch the instantiated
// graph on the caller's stream, one call for the whole batch.  The graph
// holds the images' device addresses, so a batch is re-run on new pixels by
// writing them into the same buffers.
//
// Autotuner.  For a key it has not seen on the current device, the tuner
// builds a batch of synthetic images of the size class's representative
// shape, runs the persistent kernel with each candidate tile shape, times
// the runs with CUDA events and keeps the fastest.  Results live in a
// process-wide table that ipfc_tune_save / ipfc_tune_load write to and read
// from a text file.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/ipfc.h"
#include "batch.cuh"
#include "batch_plan.h"

namespace ipfc {

int set_error(int code, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* fn);
int check_pair(const ipfc_image* src, const ipfc_image* dst, const char* fn, bool same_type);
int gaussian_taps(double sigma, int ksize, std::vector<double>& k);
bool make_sep_fast_args(const ipfc_image* src, const ipfc_image* dst, const void* in_ptr, long long in_pitch,
                        void* out_ptr, long long out_pitch, const double* kx, int kw, const double* ky, int kh, int ax,
                        int ay, int border, double delta, double bv, SepFastArgs* fp);
cudaError_t batch_launch_light(const BatchItem*, const BatchTile*, int, unsigned*, int, size_t, cudaStream_t);
cudaError_t batch_launch_mem(const BatchItem*, const BatchTile*, int, unsigned*, int, size_t, cudaStream_t);
cudaError_t batch_occupancy_light(size_t smem, int* occ);
cudaError_t batch_occupancy_mem(size_t smem, int* occ);
bool batch_sep_group_light(int k, int c, const SepGroup& g, int n, int max_tiles, cudaStream_t s, cudaError_t* e);
bool batch_sep_group_heavy(int k, int c, const SepGroup& g, int n, int max_tiles, cudaStream_t s, cudaError_t* e);

cudaError_t batch_sep_group_launch(int K, int C, const SepGroup& g, int n, int max_tiles, cudaStream_t s) {
    cudaError_t e = cudaErrorInvalidValue;
    if (n < 1 || n > kSepGroupItems || max_tiles < 1) return e;
    if (batch_sep_group_light(K, C, g, n, max_tiles, s, &e) || batch_sep_group_heavy(K, C, g, n, max_tiles, s, &e))
        return e;
    return cudaErrorInvalidValue;
}

cudaError_t batch_launch(int cls, const BatchItem* items, const BatchTile* tiles, int ntiles, unsigned* counter,
                         int grid, size_t smem, cudaStream_t s) {
    // the heavy class has no queue tiles (its separable items are group launches)
    if (cls == kBatchLight) return batch_launch_light(items, tiles, ntiles, counter, grid, smem, s);
    if (cls == kBatchMem) return batch_launch_mem(items, tiles, ntiles, counter, grid, smem, s);
    return cudaErrorInvalidValue;
}

cudaError_t batch_occupancy(int cls, size_t smem, int* occ) {
    if (cls == kBatchLight) return batch_occupancy_light(smem, occ);
    if (cls == kBatchMem) return batch_occupancy_mem(smem, occ);
    return cudaErrorInvalidValue;
}

namespace {

// ---- autotuner table ---------------------------------------------------------
struct TuneKey {
    int kind, k, c, size_class;
    bool operator<(const TuneKey& o) const {
        if (kind != o.kind) return kind < o.kind;
        if (k != o.k) return k < o.k;
        if (c != o.c) return c < o.c;
        return size_class < o.size_class;
    }
};
constexpr int kMaxDevices = 32;
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune[kMaxDevices];

// Size classes by pixel count, and the shape each class is tuned on.
constexpr int kSizeClasses = 4;
int size_class_of(int W, int H) {
    const long long px = (long long)W * H;
    return px < 65536 ? 0 : px < 524288 ? 1 : px < 2097152 ? 2 : 3;
}
const int kClassSide[kSizeClasses] = {192, 512, 1024, 2048};

std::vector<TuneVal> candidates(int kind, int k) {
    if (kind == kBatchSep) return {{2 * k, 0}, {4 * k, 0}, {8 * k, 0}, {16 * k, 0}};
    return {{128, 16}, {128, 32}, {256, 16}, {256, 32}, {256, 64}};
}

TuneVal default_val(int kind, int k) { return kind == kBatchSep ? TuneVal{8 * k, 0} : TuneVal{128, 32}; }

int batch_class(int kind, int k) {
    if (kind == kBatchSep) return k > kBatchLightMaxTaps ? kBatchHeavy : kBatchLight;
    if (kind == kBatchMedian) return (k == 3 || k == 5) ? kBatchMem : kBatchLight;
    return kBatchMem;  // morphology
}

struct Tiling {
    int cls = 0;
    int nx = 0, ny = 0;
    size_t smem = 0;
    double cost = 0;  // estimated cost of one tile (sample-operations)
};

// Applies tile parameters v to an item and describes its tiling.
Tiling tile_item(BatchItem& it, int W, int H, TuneVal v) {
    Tiling t;
    t.cls = batch_class(it.kind, it.K);
    if (it.kind == kBatchSep) {
        const int px = batch_sep_px(it.K, it.C);
        int rows = std::max(1, std::min(v.a, H));
        it.u.sep.rows_per_cta = rows;
        it.u.sep.strips = (W + px - 1) / px;
        t.nx = it.u.sep.strips;
        t.ny = (H + rows - 1) / rows;
        t.smem = batch_sep_smem(it.K, it.C);
        t.cost = (double)(2 * rows + it.K) * px * it.C * it.K;
    } else {
        it.tx = v.a;
        it.ty = v.b;
        t.nx = (W * it.C + it.tx - 1) / it.tx;
        t.ny = (H + it.ty - 1) / it.ty;
        if (it.kind == kBatchMedian) {
            t.smem = (it.K == 3 || it.K == 5) ? median_u8_tile_bytes(it.tx, it.ty, it.K, it.C)
                                              : median_tile_bytes(it.tx, it.ty, it.K, it.C);
            t.cost = (double)it.tx * it.ty * it.K * it.K * ((it.K == 3 || it.K == 5) ? 1 : 4);
        } else {
            const MorphCore& m = it.u.morph;
            t.smem = morph_u8_tile_bytes(it.tx, it.ty, m.sw, m.sh, it.C);
            t.cost = (double)it.tx * (it.ty + m.sh) * (m.sw + m.sh) / 4;
        }
    }
    return t;
}

// A plan in device memory: items, tiles (class 0 first), two counters.
struct Plan {
    HostPlan host;
    BatchItem* d_items = nullptr;
    BatchTile* d_tiles = nullptr;
    unsigned* d_counter = nullptr;
    int grid[kBatchClasses] = {};

    void release() {
        if (d_items) cudaFree(d_items);
        if (d_tiles) cudaFree(d_tiles);
        if (d_counter) cudaFree(d_counter);
        d_items = nullptr;
        d_tiles = nullptr;
        d_counter = nullptr;
    }
};

}  // namespace

void build_host_plan(const std::vector<HostItem>& items, const std::vector<TuneVal>& vals, HostPlan* p) {
    const int n = (int)items.size();
    p->items.resize(n);
    std::vector<Tiling> tl(n);
    std::vector<TuneVal> v(vals.begin(), vals.end());
    for (int i = 0; i < n; ++i) {
        p->items[i] = items[i].it;
        tl[i] = tile_item(p->items[i], items[i].W, items[i].H, v[i]);
    }
    // The tuned row counts suit batches of many images.  A separable class
    // whose tiles fill less than 80 % of its resident CTAs (a few large
    // images, as a server's batches often are) gets shorter tiles, down to
    // 2K rows, so that SMs do not idle.
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                   cudaSuccess)
        cudaGetLastError();
    const int slots[kBatchClasses] = {2 * sms, sms, 4 * sms};  // resident CTAs per class (registers bound)
    for (int c : {kBatchLight, kBatchHeavy}) {
        for (int round = 0; round < 4 && sms > 0; ++round) {
            long long tiles = 0;
            for (int i = 0; i < n; ++i)
                if (tl[i].cls == c && items[i].W > 0 && items[i].H > 0) tiles += (long long)tl[i].nx * tl[i].ny;
            if (tiles == 0 || 5 * tiles >= 4 * (long long)slots[c]) break;  // at least 80 % of the slots busy
            bool shrunk = false;
            for (int i = 0; i < n; ++i) {
                if (tl[i].cls != c || items[i].it.kind != kBatchSep) continue;
                const int k = items[i].it.K, rows = std::min(v[i].a, items[i].H);
                if (rows <= 2 * k) continue;
                v[i].a = std::max(2 * k, rows / 2);
                p->items[i] = items[i].it;
                tl[i] = tile_item(p->items[i], items[i].W, items[i].H, v[i]);
                shrunk = true;
            }
            if (!shrunk) break;
        }
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        if (tl[x].cls != tl[y].cls) return tl[x].cls < tl[y].cls;
        return tl[x].cost > tl[y].cost;
    });
    p->tiles.clear();
    for (int c = 0; c < kBatchClasses; ++c) {
        p->tile_off[c] = (int)p->tiles.size();
        p->smem[c] = 0;
        p->cost[c] = 0;
        p->sep_tiles[c] = 0;
        for (int i : order) {
            if (tl[i].cls != c || items[i].W == 0 || items[i].H == 0) continue;
            if (items[i].it.kind == kBatchSep) {
                p->sep_tiles[c] += tl[i].nx * tl[i].ny;
                continue;  // a group launch (below)
            }
            p->smem[c] = std::max(p->smem[c], tl[i].smem);
            for (int y = 0; y < tl[i].ny; ++y)
                for (int x = 0; x < tl[i].nx; ++x) {
                    p->tiles.push_back(BatchTile{i, x, y, 0});
                    p->cost[c] += tl[i].cost;
                }
        }
        p->ntiles[c] = (int)p->tiles.size() - p->tile_off[c];
    }
    // separable groups: same (K, C), heavy class first, each group's items in
    // the longest-first order, at most kSepGroupItems per launch
    p->groups.clear();
    for (int c : {kBatchHeavy, kBatchLight}) {
        std::vector<SepGroupLaunch> open;  // the group being filled for each (K, C)
        for (int i : order) {
            if (tl[i].cls != c || items[i].it.kind != kBatchSep || items[i].W == 0 || items[i].H == 0) continue;
            const int K = items[i].it.K, C = items[i].it.C;
            SepGroupLaunch* gr = nullptr;
            for (SepGroupLaunch& o : open)
                if (o.K == K && o.C == C) gr = &o;
            if (!gr) {
                open.push_back(SepGroupLaunch{});
                gr = &open.back();
                gr->K = K;
                gr->C = C;
                gr->cls = c;
            }
            gr->items.push_back(i);
            gr->max_tiles = std::max(gr->max_tiles, tl[i].nx * tl[i].ny);
            gr->cost += tl[i].cost * tl[i].nx * tl[i].ny;
            if ((int)gr->items.size() == kSepGroupItems) {
                p->groups.push_back(*gr);
                *gr = SepGroupLaunch{};
                gr->K = K;
                gr->C = C;
                gr->cls = c;
            }
        }
        for (const SepGroupLaunch& o : open)
            if (!o.items.empty()) p->groups.push_back(o);
    }
}

cudaError_t plan_grids(const HostPlan& p, int grid[kBatchClasses]) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (int c = 0; c < kBatchClasses && e == cudaSuccess; ++c) {
        grid[c] = 0;
        if (p.ntiles[c] == 0) continue;
        int occ = 0;
        e = batch_occupancy(c, p.smem[c], &occ);
        if (e != cudaSuccess) break;
        if (occ < 1) return cudaErrorInvalidConfiguration;
        grid[c] = std::min(sms * occ, p.ntiles[c]);
    }
    return e;
}

cudaError_t launch_plan(const BatchItem* d_items, const BatchTile* d_tiles, unsigned* d_counter, const HostPlan& p,
                        const int grid[kBatchClasses], cudaStream_t s0, const cudaStream_t* side, int nside,
                        cudaEvent_t fork, cudaEvent_t join) {
    cudaError_t e = cudaMemsetAsync(d_counter, 0, sizeof(unsigned) * kBatchClasses, s0);
    if (e != cudaSuccess) return e;
    // Work units: each separable group launch and each non-empty queue
    // kernel, with its estimated cost.  Every group launch ends with a tail of
    // uneven tiles, so with side streams the units are spread over parallel
    // lanes (largest first, each to the least-loaded lane) and the tails of
    // one launch overlap the work of others.  Without side streams the units
    // run on s0: heavy groups, the memory-bound queue, light groups, the
    // light queue.
    struct Unit {
        int group;  // index into p.groups, or -1 - class for a queue kernel
        double cost;
    };
    std::vector<Unit> units;
    for (int cls : {kBatchHeavy, kBatchLight}) {
        for (size_t g = 0; g < p.groups.size(); ++g)
            if (p.groups[g].cls == cls) units.push_back(Unit{(int)g, p.groups[g].cost});
        if (cls == kBatchHeavy) {
            for (int c : {kBatchHeavy, kBatchMem})
                if (p.ntiles[c] > 0) units.push_back(Unit{-1 - c, p.cost[c]});
        }
    }
    if (p.ntiles[kBatchLight] > 0) units.push_back(Unit{-1 - kBatchLight, p.cost[kBatchLight]});
    const int nl = (side && nside > 0 && fork && join && units.size() > 1)
                       ? 1 + std::min(nside, (int)units.size() - 1)
                       : 1;
    std::vector<cudaStream_t> lane(nl, s0);
    for (int l = 1; l < nl; ++l) lane[l] = side[l - 1];
    std::vector<int> of(units.size(), 0);
    if (nl > 1) {
        std::vector<size_t> order(units.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t x, size_t y) { return units[x].cost > units[y].cost; });
        std::vector<double> load(nl, 0.0);
        for (size_t i : order) {
            int best = 0;
            for (int l = 1; l < nl; ++l)
                if (load[l] < load[best]) best = l;
            of[i] = best;
            load[best] += units[i].cost;
        }
        // the fork follows the counter reset and precedes every launch
        if ((e = cudaEventRecord(fork, s0)) != cudaSuccess) return e;
    }
    int forked = 1;  // lanes that wait on the fork; lane 0 is s0 itself
    while (forked < nl && (e = cudaStreamWaitEvent(lane[forked], fork, 0)) == cudaSuccess) ++forked;
    SepGroup g{};  // slots past a group's items are never read
    for (size_t i = 0; i < units.size() && e == cudaSuccess; ++i) {
        cudaStream_t s = lane[of[i]];
        if (units[i].group >= 0) {
            const SepGroupLaunch& gl = p.groups[units[i].group];
            for (size_t j = 0; j < gl.items.size(); ++j) g.it[j] = p.items[gl.items[j]].u.sep;
            e = batch_sep_group_launch(gl.K, gl.C, g, (int)gl.items.size(), gl.max_tiles, s);
        } else {
            const int c = -1 - units[i].group;
            e = batch_launch(c, d_items, d_tiles + p.tile_off[c], p.ntiles[c], d_counter + c, grid[c], p.smem[c], s);
        }
    }
    // Join every forked lane, after an error too, so that a stream capture
    // in progress ends with all its branches merged back into s0: s0 waits
    // for each lane (the event is re-recorded per lane).
    for (int l = 1; l < forked; ++l) {
        cudaError_t j = cudaEventRecord(join, lane[l]);
        if (j == cudaSuccess) j = cudaStreamWaitEvent(s0, join, 0);
        if (e == cudaSuccess) e = j;
    }
    return e;
}

TuneVal tuned_or_default(int kind, int k, int c, int W, int H) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= kMaxDevices) {
        cudaGetLastError();
        return default_val(kind, k);
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto f = g_tune[dev].find(TuneKey{kind, k, c, size_class_of(W, H)});
    return f != g_tune[dev].end() ? f->second : default_val(kind, k);
}

namespace {

cudaError_t make_plan(const std::vector<HostItem>& items, const std::vector<TuneVal>& vals, Plan* p) {
    build_host_plan(items, vals, &p->host);
    const HostPlan& h = p->host;
    cudaError_t e = plan_grids(h, p->grid);
    if (e != cudaSuccess) return e;
    const size_t n = h.items.size();
    if (n > 0) e = cudaMalloc((void**)&p->d_items, sizeof(BatchItem) * n);
    if (e == cudaSuccess && !h.tiles.empty()) e = cudaMalloc((void**)&p->d_tiles, sizeof(BatchTile) * h.tiles.size());
    if (e == cudaSuccess) e = cudaMalloc((void**)&p->d_counter, sizeof(unsigned) * kBatchClasses);
    if (e == cudaSuccess && n > 0)
        e = cudaMemcpy(p->d_items, h.items.data(), sizeof(BatchItem) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !h.tiles.empty())
        e = cudaMemcpy(p->d_tiles, h.tiles.data(), sizeof(BatchTile) * h.tiles.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) p->release();
    return e;
}

// Enqueues one execution of a plan: counter reset, then the classes' kernels
// (on s0, or as parallel branches when s1, s2 and the events are given).
cudaError_t enqueue_plan(const Plan& p, cudaStream_t s0, const cudaStream_t* side, int nside, cudaEvent_t fork,
                         cudaEvent_t join) {
    return launch_plan(p.d_items, p.d_tiles, p.d_counter, p.host, p.grid, s0, side, nside, fork, join);
}

// Times candidate tile shapes for one key on synthetic images; returns the
// fastest.
cudaError_t tune_key(const TuneKey& key, const HostItem& proto, TuneVal* best) {
    const int side = kClassSide[key.size_class];
    const int W = side, H = side, C = key.c;
    const long long bytes = (long long)W * H * C;
    // Enough copies to fill the device several times over, each with its own
    // source and destination: the 256 MB or more they span is beyond L2, so
    // memory-bound tiles are timed reading DRAM as a real batch does.
    const int copies = (int)std::max(4LL, std::min(1024LL, (256LL << 20) / std::max(1LL, bytes)));
    unsigned char* buf = nullptr;
    cudaError_t e = cudaMalloc((void**)&buf, (size_t)bytes * 2 * copies);
    if (e != cudaSuccess) return e;
    cudaStream_t s = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    e = cudaMemset(buf, 0x5a, (size_t)bytes * 2 * copies);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    std::vector<HostItem> items((size_t)copies, proto);
    for (size_t i = 0; i < items.size(); ++i) {
        HostItem& h = items[i];
        h.W = W;
        h.H = H;
        BatchItem& it = h.it;
        unsigned char* src = buf + (size_t)bytes * 2 * i;  // only the time is used
        unsigned char* dst = src + bytes;
        if (it.kind == kBatchSep) {
            it.u.sep.src = src;
            it.u.sep.spitch = (long long)W * C;
            it.u.sep.dst = dst;
            it.u.sep.dpitch = (long long)W * C;
            it.u.sep.W = W;
            it.u.sep.H = H;
            it.u.sep.vec_load = 1;
            it.u.sep.vec_store = ((W * C) % 16 == 0) ? 1 : 0;
        } else if (it.kind == kBatchMedian) {
            it.u.med.src = src;
            it.u.med.spitch = (long long)W * C;
            it.u.med.dst = dst;
            it.u.med.dpitch = (long long)W * C;
            it.u.med.W = W;
            it.u.med.H = H;
        } else {
            it.u.morph.src = src;
            it.u.morph.spitch = (long long)W * C;
            it.u.morph.dst = dst;
            it.u.morph.dpitch = (long long)W * C;
            it.u.morph.W = W;
            it.u.morph.H = H;
        }
    }
    float best_ms = 1e30f;
    *best = default_val(key.kind, key.k);
    for (const TuneVal& v : candidates(key.kind, key.k)) {
        if (e != cudaSuccess) break;
        if (key.kind != kBatchSep) {
            const size_t need = key.kind == kBatchMedian
                                    ? ((key.k == 3 || key.k == 5) ? median_u8_tile_bytes(v.a, v.b, key.k, C)
                                                                  : median_tile_bytes(v.a, v.b, key.k, C))
                                    : morph_u8_tile_bytes(v.a, v.b, proto.it.u.morph.sw, proto.it.u.morph.sh, C);
            if (need > 96 * 1024) continue;
        }
        std::vector<TuneVal> vals((size_t)copies, v);
        Plan p;
        e = make_plan(items, vals, &p);
        if (e != cudaSuccess) break;
        float ms = 1e30f;
        for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
            e = cudaEventRecord(t0, s);
            if (e == cudaSuccess) e = enqueue_plan(p, s, nullptr, 0, nullptr, nullptr);
            if (e == cudaSuccess) e = cudaEventRecord(t1, s);
            if (e == cudaSuccess) e = cudaEventSynchronize(t1);
            float m = 0;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&m, t0, t1);
            if (rep > 0) ms = std::min(ms, m);  // the first run warms up
        }
        p.release();
        if (e == cudaSuccess && ms < best_ms) {
            best_ms = ms;
            *best = v;
        }
    }
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (s) cudaStreamDestroy(s);
    cudaFree(buf);
    return e;
}

bool tune_env_disabled() {
    const char* v = std::getenv("IPFC_AUTOTUNE");
    return v && std::strcmp(v, "0") == 0;
}

}  // namespace

}  // namespace ipfc

using namespace ipfc;

struct ipfc_batch {
    std::vector<HostItem> items;
    int autotune = 1;
    int use_graph = 1;
    int device = -1;
    bool planned = false;
    Plan plan;
    static constexpr int kLanes = 8;
    cudaStream_t st[kLanes] = {};  // capture stream and the branches
    cudaEvent_t ev[2] = {nullptr, nullptr};            // fork, join
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    void drop_plan() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        plan.release();
        planned = false;
    }
    ~ipfc_batch() {
        drop_plan();
        for (int i = 0; i < kLanes; ++i)
            if (st[i]) cudaStreamDestroy(st[i]);
        for (int i = 0; i < 2; ++i)
            if (ev[i]) cudaEventDestroy(ev[i]);
    }
};

namespace {

int batch_common(ipfc_batch* b, const ipfc_image* src, const ipfc_image* dst, const char* fn) {
    if (!b) return set_error(IPFC_ERR_INVALID, "ipf: %s: null batch", fn);
    if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
    if (src->mem != IPFC_MEM_DEVICE || dst->mem != IPFC_MEM_DEVICE)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: batched images must be in device memory", fn);
    if (src->dtype != IPFC_U8 || dst->dtype != IPFC_U8)
        return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: batches take uint8 images", fn);
    if (src->channels != 1 && src->channels != 3 && src->channels != 4)
        return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: batches take 1, 3 or 4 channels", fn);
    int rc = check_pair(src, dst, fn, false);
    if (rc > 0) return rc;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, fn);
    if (b->device < 0) b->device = dev;
    if (b->device != dev) return set_error(IPFC_ERR_INVALID, "ipf: %s: batch belongs to device %d", fn, b->device);
    return rc;  // 0, or -1 for an empty image
}

long long pitch_or_dense(const ipfc_image* im) {
    return im->pitch > 0 ? im->pitch : (long long)im->width * im->channels;
}

void add_item(ipfc_batch* b, const BatchItem& it, int W, int H) {
    HostItem h;
    h.it = it;
    h.W = W;
    h.H = H;
    b->items.push_back(h);
    b->drop_plan();
}

int add_sep(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, const double* kx, int kw, const double* ky, int kh,
            int border, double delta, double bv, const char* fn) {
    if (!kx || !ky || kw <= 0 || kh <= 0) return set_error(IPFC_ERR_INVALID, "ipf: separable filter: empty kernel");
    if (border < IPFC_BORDER_CONSTANT || border > IPFC_BORDER_WRAP)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid border mode", fn);
    int rc = batch_common(b, src, dst, fn);
    if (rc > 0) return rc;
    if (kw != kh || kw % 2 == 0 || kw < 3 || kw > kBatchMaxTaps)
        return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: batches take equal odd tap counts from 3 to %d", fn,
                         kBatchMaxTaps);
    BatchItem it;
    std::memset(&it, 0, sizeof(it));
    it.kind = kBatchSep;
    it.K = kw;
    it.C = src->channels;
    if (rc == 0 && !make_sep_fast_args(src, dst, src->data, pitch_or_dense(src), dst->data, pitch_or_dense(dst), kx, kw,
                                       ky, kh, kw / 2, kh / 2, border, delta, bv, &it.u.sep))
        return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: taps not covered by the batched kernel", fn);
    add_item(b, it, rc == 0 ? src->width : 0, rc == 0 ? src->height : 0);
    return IPFC_OK;
}

int plan_batch(ipfc_batch* b, const char* fn) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, fn);
    if (dev >= kMaxDevices) return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: device index %d out of range", fn, dev);
    std::vector<TuneVal> vals(b->items.size());
    const bool tune = b->autotune && !tune_env_disabled();
    for (size_t i = 0; i < b->items.size(); ++i) {
        const HostItem& h = b->items[i];
        const TuneKey key{h.it.kind, h.it.K, h.it.C, size_class_of(h.W, h.H)};
        TuneVal v = default_val(key.kind, key.k);
        bool found = false;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto f = g_tune[dev].find(key);
            if (f != g_tune[dev].end()) {
                v = f->second;
                found = true;
            }
        }
        if (!found && tune && h.W > 0) {
            e = tune_key(key, h, &v);
            if (e != cudaSuccess) return cuda_status(e, fn);
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune[dev][key] = v;
        }
        vals[i] = v;
    }
    e = make_plan(b->items, vals, &b->plan);
    if (e != cudaSuccess) return cuda_status(e, fn);
    for (int i = 0; i < ipfc_batch::kLanes && e == cudaSuccess; ++i)
        if (!b->st[i]) e = cudaStreamCreateWithFlags(&b->st[i], cudaStreamNonBlocking);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i)
        if (!b->ev[i]) e = cudaEventCreateWithFlags(&b->ev[i], cudaEventDisableTiming);
    if (e == cudaSuccess && b->use_graph) {
        e = cudaStreamBeginCapture(b->st[0], cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t e2 = enqueue_plan(b->plan, b->st[0], b->st + 1, ipfc_batch::kLanes - 1, b->ev[0], b->ev[1]);
            e = cudaStreamEndCapture(b->st[0], &b->graph);
            if (e2 != cudaSuccess) e = e2;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    }
    if (e != cudaSuccess) {
        b->drop_plan();
        return cuda_status(e, fn);
    }
    b->planned = true;
    return IPFC_OK;
}

}  // namespace

extern "C" {

int ipfc_batch_create(ipfc_batch** out) {
    if (!out) return set_error(IPFC_ERR_INVALID, "ipf: batch: null output pointer");
    *out = new ipfc_batch();
    return IPFC_OK;
}

int ipfc_batch_destroy(ipfc_batch* b) {
    delete b;
    return IPFC_OK;
}

int ipfc_batch_set_option(ipfc_batch* b, int option, int value) {
    if (!b) return set_error(IPFC_ERR_INVALID, "ipf: batch: null batch");
    if (option == IPFC_BATCH_AUTOTUNE) b->autotune = value ? 1 : 0;
    else if (option == IPFC_BATCH_GRAPH) b->use_graph = value ? 1 : 0;
    else return set_error(IPFC_ERR_INVALID, "ipf: batch: unknown option %d", option);
    b->drop_plan();
    return IPFC_OK;
}

int ipfc_batch_add_sep_filter(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, const double* kx, int kw,
                              const double* ky, int kh, int border, double delta, double border_value) {
    return add_sep(b, src, dst, kx, kw, ky, kh, border, delta, border_value, "sepFilter2D (batch)");
}

int ipfc_batch_add_gaussian_blur(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, double sigma_x,
                                 double sigma_y, int ksize, int border) {
    if (sigma_y <= 0) sigma_y = sigma_x;
    std::vector<double> kx, ky;
    if (gaussian_taps(sigma_x, ksize, kx)) return IPFC_ERR_INVALID;
    if (gaussian_taps(sigma_y, ksize, ky)) return IPFC_ERR_INVALID;
    return add_sep(b, src, dst, kx.data(), (int)kx.size(), ky.data(), (int)ky.size(), border, 0.0, 0.0,
                   "gaussianBlur (batch)");
}

int ipfc_batch_add_median_blur(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, int ksize, int border) {
    const char* fn = "medianBlur (batch)";
    if (!(ksize >= 1 && ksize % 2 == 1))
        return set_error(IPFC_ERR_INVALID, "ipf: medianBlur: ksize must be odd and positive");
    if (border == IPFC_BORDER_CONSTANT)
        return set_error(IPFC_ERR_INVALID, "ipf: medianBlur: Constant border is not supported");
    if (border < IPFC_BORDER_CONSTANT || border > IPFC_BORDER_WRAP)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid border mode", fn);
    int rc = batch_common(b, src, dst, fn);
    if (rc > 0) return rc;
    if (ksize < 3 || ksize > 15)
        return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: batches take ksize 3 to 15 (ksize 1 is a copy)", fn);
    BatchItem it;
    std::memset(&it, 0, sizeof(it));
    it.kind = kBatchMedian;
    it.K = ksize;
    it.C = src->channels;
    it.u.med = MedianArgs{src->data, pitch_or_dense(src), dst->data, pitch_or_dense(dst), src->width, src->height,
                          src->channels, ksize, border};
    add_item(b, it, rc == 0 ? src->width : 0, rc == 0 ? src->height : 0);
    return IPFC_OK;
}

static int batch_morph(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, const uint8_t* se, int sw, int sh,
                       int iterations, bool is_min) {
    const char* fn = is_min ? "erode (batch)" : "dilate (batch)";
    if (!se || sw <= 0 || sh <= 0)
        return set_error(IPFC_ERR_INVALID,
                         "ipf: morphology: structuring element must be a non-empty single-channel mask");
    int rc = batch_common(b, src, dst, fn);
    if (rc > 0) return rc;
    for (int i = 0; i < sw * sh; ++i)
        if (!se[i]) return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: batches take all-ones (Rect) elements", fn);
    if (iterations != 1) return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: batches take one iteration", fn);
    if (sw > 31 || sh > 31) return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: batches take elements up to 31x31", fn);
    BatchItem it;
    std::memset(&it, 0, sizeof(it));
    it.kind = kBatchMorph;
    it.K = sw;
    it.C = src->channels;
    MorphCore& m = it.u.morph;
    m.src = src->data;
    m.spitch = pitch_or_dense(src);
    m.dst = dst->data;
    m.dpitch = pitch_or_dense(dst);
    m.W = src->width;
    m.H = src->height;
    m.C = src->channels;
    m.sw = sw;
    m.sh = sh;
    m.ax = sw / 2;
    m.ay = sh / 2;
    m.is_rect = 1;
    m.is_min = is_min ? 1 : 0;
    m.noffs = sw * sh;
    add_item(b, it, rc == 0 ? src->width : 0, rc == 0 ? src->height : 0);
    return IPFC_OK;
}

int ipfc_batch_add_erode(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, const uint8_t* se, int se_w, int se_h,
                         int iterations) {
    return batch_morph(b, src, dst, se, se_w, se_h, iterations, true);
}

int ipfc_batch_add_dilate(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, const uint8_t* se, int se_w,
                          int se_h, int iterations) {
    return batch_morph(b, src, dst, se, se_w, se_h, iterations, false);
}

int ipfc_batch_run(ipfc_batch* b, void* stream) {
    const char* fn = "batch";
    if (!b) return set_error(IPFC_ERR_INVALID, "ipf: batch: null batch");
    if (b->items.empty()) return IPFC_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, fn);
    if (dev != b->device) return set_error(IPFC_ERR_INVALID, "ipf: batch: batch belongs to device %d", b->device);
    if (!b->planned) {
        int rc = plan_batch(b, fn);
        if (rc) return rc;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (b->exec) {
        e = cudaGraphLaunch(b->exec, s);
    } else {
        e = enqueue_plan(b->plan, s, nullptr, 0, nullptr, nullptr);
    }
    return e == cudaSuccess ? IPFC_OK : cuda_status(e, fn);
}

int ipfc_batch_info(const ipfc_batch* b, int what, long long* value) {
    if (!b || !value) return set_error(IPFC_ERR_INVALID, "ipf: batch: null argument");
    const Plan& p = b->plan;
    switch (what) {
        case IPFC_BATCH_INFO_ITEMS: *value = (long long)b->items.size(); break;
        case IPFC_BATCH_INFO_PLANNED: *value = b->planned ? 1 : 0; break;
        case IPFC_BATCH_INFO_TILES_LIGHT: *value = p.host.ntiles[kBatchLight] + p.host.sep_tiles[kBatchLight]; break;
        case IPFC_BATCH_INFO_TILES_HEAVY: *value = p.host.ntiles[kBatchHeavy] + p.host.sep_tiles[kBatchHeavy]; break;
        case IPFC_BATCH_INFO_TILES_MEM: *value = p.host.ntiles[kBatchMem]; break;
        case IPFC_BATCH_INFO_GRID_LIGHT: *value = p.grid[kBatchLight]; break;
        case IPFC_BATCH_INFO_GRID_HEAVY: *value = p.grid[kBatchHeavy]; break;
        case IPFC_BATCH_INFO_GRID_MEM: *value = p.grid[kBatchMem]; break;
        case IPFC_BATCH_INFO_KERNELS:  // kernel launches per run: queue classes and separable groups
            *value = (long long)p.host.groups.size();
            for (int c = 0; c < kBatchClasses; ++c) *value += p.host.ntiles[c] > 0;
            break;
        case IPFC_BATCH_INFO_GRAPH: *value = b->exec ? 1 : 0; break;
        default: return set_error(IPFC_ERR_INVALID, "ipf: batch: unknown info %d", what);
    }
    return IPFC_OK;
}

int ipfc_tune_get(int op, int k, int channels, int size_class, int* a, int* b) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= kMaxDevices) {
        cudaGetLastError();
        dev = 0;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto f = g_tune[dev].find(TuneKey{op, k, channels, size_class});
    if (f == g_tune[dev].end()) return set_error(IPFC_ERR_INVALID, "ipf: tune: no entry");
    if (a) *a = f->second.a;
    if (b) *b = f->second.b;
    return IPFC_OK;
}

int ipfc_tune_set(int op, int k, int channels, int size_class, int a, int b) {
    if (op < kBatchSep || op > kBatchMorph || size_class < 0 || size_class >= kSizeClasses || a <= 0 ||
        (op != kBatchSep && b <= 0))
        return set_error(IPFC_ERR_INVALID, "ipf: tune: invalid entry");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= kMaxDevices) {
        cudaGetLastError();
        dev = 0;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[dev][TuneKey{op, k, channels, size_class}] = TuneVal{a, b};
    return IPFC_OK;
}

int ipfc_tune_save(const char* path) {
    if (!path) return set_error(IPFC_ERR_INVALID, "ipf: tune: null path");
    FILE* f = std::fopen(path, "w");
    if (!f) return set_error(IPFC_ERR_INVALID, "ipf: tune: cannot write %s", path);
    std::fprintf(f, "# ipfc autotune table: device op k channels size_class a b\n");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (int d = 0; d < kMaxDevices; ++d)
        for (const auto& kv : g_tune[d])
            std::fprintf(f, "%d %d %d %d %d %d %d\n", d, kv.first.kind, kv.first.k, kv.first.c, kv.first.size_class,
                         kv.second.a, kv.second.b);
    std::fclose(f);
    return IPFC_OK;
}

int ipfc_tune_load(const char* path, int* count) {
    if (!path) return set_error(IPFC_ERR_INVALID, "ipf: tune: null path");
    FILE* f = std::fopen(path, "r");
    if (!f) return set_error(IPFC_ERR_INVALID, "ipf: tune: cannot read %s", path);
    char line[256];
    int n = 0;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    while (std::fgets(line, sizeof(line), f)) {
        if (line[0] == '#') continue;
        int d, op, k, c, sc, a, b;
        if (std::sscanf(line, "%d %d %d %d %d %d %d", &d, &op, &k, &c, &sc, &a, &b) != 7) continue;
        if (d < 0 || d >= kMaxDevices || sc < 0 || sc >= kSizeClasses || a <= 0) continue;
        g_tune[d][TuneKey{op, k, c, sc}] = TuneVal{a, b};
        ++n;
    }
    std::fclose(f);
    if (count) *count = n;
    return IPFC_OK;
}

int ipfc_tune_clear(void) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (int d = 0; d < kMaxDevices; ++d) g_tune[d].clear();
    return IPFC_OK;
}

}  // extern "C"
