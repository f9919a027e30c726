// serve.cu -- the request server (ipfc_server_*): continuous batching of
// filter requests against a device-memory budget.
//
// Requests (one image and one op each, host or device images) are queued by
// ipfc_server_submit with an arrival time.  One scheduler thread per server
// loops over three steps, without waiting for the device in between:
//  1. completion: every in-flight group whose event has fired is retired --
//     its requests' device memory and slots return to the budget and their
//     completions (arrival, admission and completion times) are published;
//  2. admission: pending requests whose arrival time has come are admitted
//     in arrival order while a slot is free and their device bytes fit in
//     what the budget has left (a request larger than the whole budget
//     fails); admission never waits for running work, so requests arriving
//     while others run are admitted as soon as slots and memory free up;
//  3. dispatch: the admitted requests are spread round-robin over the
//     server's streams.  On each stream: device buffers from the server's
//     memory pool, host->device copies, then the kernels -- requests the
//     batch kernels cover (uint8 gaussianBlur up to 25 taps, medianBlur,
//     erode/dilate by a rect) merged into one direct launch of the
//     persistent tile-queue kernels, the others one launch each through the
//     per-image entry points -- then device->host copies, stream-ordered
//     frees and the group's completion event.
// Work of different groups overlaps on the device (separate streams), and
// each request runs the same kernel code as its per-image call, so its
// result does not depend on what else is in flight.
//
// Device memory comes from a dedicated stream-ordered pool whose release
// threshold is the budget: images and plans stay in device memory that the
// pool keeps mapped, not in per-request cudaMalloc/cudaFree.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/ipfc.h"
#include "batch_plan.h"

namespace ipfc {
int set_error(int code, const char* fmt, ...);
void set_shared_gpu(bool on);
int cuda_status(cudaError_t e, const char* fn);
size_t elem_bytes(int dt);
int gaussian_taps(double sigma, int ksize, std::vector<double>& k);
bool make_sep_fast_args(const ipfc_image* src, const ipfc_image* dst, const void* in_ptr, long long in_pitch,
                        void* out_ptr, long long out_pitch, const double* kx, int kw, const double* ky, int kh, int ax,
                        int ay, int border, double delta, double bv, SepFastArgs* fp);
}  // namespace ipfc

using namespace ipfc;

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
    ipfc_request r;
    std::vector<float> taps;  // filter2D taps, copied at submit
    unsigned long long ticket = 0;
    double arrival = 0, admitted = 0;
    size_t dev_bytes = 0;
    int status = IPFC_OK;
    // device views while in flight
    void* dsrc = nullptr;
    void* ddst = nullptr;
    long long dspitch = 0, ddpitch = 0;
};

struct Group {
    std::vector<Req> reqs;
    cudaEvent_t done = nullptr;
};

long long row_bytes_of(const ipfc_image& im) {
    return (long long)im.width * im.channels * (long long)elem_bytes(im.dtype);
}
long long pitch_of_img(const ipfc_image& im) { return im.pitch > 0 ? im.pitch : row_bytes_of(im); }
size_t round256(size_t v) { return (v + 255) / 256 * 256; }

size_t request_bytes(const ipfc_request& r) {
    size_t b = 0;
    if (r.src.mem == IPFC_MEM_HOST) b += round256((size_t)row_bytes_of(r.src) * r.src.height);
    if (r.dst.mem == IPFC_MEM_HOST) b += round256((size_t)row_bytes_of(r.dst) * r.dst.height);
    if (r.op == IPFC_OP_FILTER2D) b += round256((size_t)r.kw * r.kh * 16);
    return b + 4096;  // batch plan share
}

}  // namespace

struct ipfc_server {
    ipfc_server_config cfg;
    int device = 0;
    cudaMemPool_t pool = nullptr;
    std::vector<cudaStream_t> streams;
    int next_stream = 0;
    Clock::time_point epoch;

    std::mutex mu;
    std::condition_variable cv_submit, cv_done;
    std::deque<Req> pending;
    std::deque<ipfc_completion> completions;
    unsigned long long next_ticket = 1;
    unsigned long long submitted = 0, finished = 0;
    bool stop = false;

    // scheduler-owned
    std::vector<Group> inflight;
    size_t used_bytes = 0;
    int used_slots = 0;
    std::thread worker;

    // injected allocation failure: the n-th device-buffer allocation of a
    // request (1-based, counted by the scheduler) fails (0: none)
    std::atomic<long long> fail_alloc_nth{0};
    long long allocs = 0;

    // statistics
    std::atomic<long long> st_groups{0}, st_batched{0}, st_batch_launches{0}, st_max_slots{0}, st_failed{0};
    std::atomic<long long> st_max_bytes{0};

    double now() const { return std::chrono::duration<double>(Clock::now() - epoch).count(); }
};

namespace {

void complete_group(ipfc_server* s, Group& g) {
    const double t = s->now();
    std::lock_guard<std::mutex> lk(s->mu);
    for (Req& q : g.reqs) {
        ipfc_completion c;
        c.ticket = q.ticket;
        c.status = q.status;
        c.arrival = q.arrival;
        c.admitted = q.admitted;
        c.done = t;
        s->completions.push_back(c);
        if (q.status != IPFC_OK) s->st_failed++;
        s->used_bytes -= q.dev_bytes;
        s->used_slots -= 1;
        s->finished++;
    }
    s->cv_done.notify_all();
}

// Whether the batch kernels cover a request.
bool batchable(const ipfc_request& r) {
    if (r.src.dtype != IPFC_U8 || r.dst.dtype != IPFC_U8) return false;
    if (r.src.channels != 1 && r.src.channels != 3 && r.src.channels != 4) return false;
    if (r.src.width == 0 || r.src.height == 0) return false;
    if (r.op == IPFC_OP_GAUSSIAN) {
        const double sy = r.sigma_y > 0 ? r.sigma_y : r.sigma_x;
        int k = r.ksize;
        if (k <= 0) {
            if (!(r.sigma_x > 0) || !(sy > 0)) return false;
            const int rx = static_cast<int>(3.0 * r.sigma_x + 0.5), ry = static_cast<int>(3.0 * sy + 0.5);
            const int kx = 2 * (rx > 1 ? rx : 1) + 1, ky = 2 * (ry > 1 ? ry : 1) + 1;
            if (kx != ky) return false;
            k = kx;
        }
        return k >= 3 && k <= kBatchMaxTaps && k % 2 == 1 && r.border >= 0 && r.border <= 4;
    }
    if (r.op == IPFC_OP_MEDIAN) return r.ksize >= 3 && r.ksize <= 15 && r.ksize % 2 == 1 && r.border >= 1 && r.border <= 4;
    if (r.op == IPFC_OP_ERODE || r.op == IPFC_OP_DILATE) return r.ksize >= 1 && r.ksize <= 31;
    return false;
}

// Builds the batch item of a batchable request on its device views.
bool batch_item(const Req& q, HostItem* h) {
    const ipfc_request& r = q.r;
    ipfc_image sv = r.src, dv = r.dst;
    sv.data = q.dsrc;
    sv.pitch = q.dspitch;
    sv.mem = IPFC_MEM_DEVICE;
    dv.data = q.ddst;
    dv.pitch = q.ddpitch;
    dv.mem = IPFC_MEM_DEVICE;
    BatchItem& it = h->it;
    std::memset(&it, 0, sizeof(it));
    it.C = sv.channels;
    h->W = sv.width;
    h->H = sv.height;
    if (r.op == IPFC_OP_GAUSSIAN) {
        std::vector<double> kx, ky;
        const double sy = r.sigma_y > 0 ? r.sigma_y : r.sigma_x;
        if (gaussian_taps(r.sigma_x, r.ksize, kx) || gaussian_taps(sy, r.ksize, ky)) return false;
        it.kind = kBatchSep;
        it.K = (int)kx.size();
        return make_sep_fast_args(&sv, &dv, sv.data, sv.pitch, dv.data, dv.pitch, kx.data(), (int)kx.size(),
                                  ky.data(), (int)ky.size(), (int)kx.size() / 2, (int)ky.size() / 2, r.border, 0.0,
                                  0.0, &it.u.sep);
    }
    if (r.op == IPFC_OP_MEDIAN) {
        it.kind = kBatchMedian;
        it.K = r.ksize;
        it.u.med = MedianArgs{sv.data, sv.pitch, dv.data, dv.pitch, sv.width, sv.height, sv.channels, r.ksize,
                              r.border};
        return true;
    }
    it.kind = kBatchMorph;
    it.K = r.ksize;
    MorphCore& m = it.u.morph;
    m.src = sv.data;
    m.spitch = sv.pitch;
    m.dst = dv.data;
    m.dpitch = dv.pitch;
    m.W = sv.width;
    m.H = sv.height;
    m.C = sv.channels;
    m.sw = m.sh = r.ksize;
    m.ax = m.ay = r.ksize / 2;
    m.is_rect = 1;
    m.is_min = r.op == IPFC_OP_ERODE ? 1 : 0;
    m.noffs = r.ksize * r.ksize;
    return true;
}

// Runs one non-batched request through its per-image entry point.
int run_single(const Req& q, cudaStream_t st) {
    // leave SMs to the other streams' requests (no persistent whole-GPU kernel)
    struct SharedGpu {
        SharedGpu() { set_shared_gpu(true); }
        ~SharedGpu() { set_shared_gpu(false); }
    } shared_gpu;
    const ipfc_request& r = q.r;
    ipfc_image sv = r.src, dv = r.dst;
    sv.data = q.dsrc;
    sv.pitch = q.dspitch;
    sv.mem = IPFC_MEM_DEVICE;
    dv.data = q.ddst;
    dv.pitch = q.ddpitch;
    dv.mem = IPFC_MEM_DEVICE;
    switch (r.op) {
        case IPFC_OP_GAUSSIAN:
            return ipfc_gaussian_blur(&sv, &dv, r.sigma_x, r.sigma_y, r.ksize, r.border, st);
        case IPFC_OP_SOBEL: return ipfc_sobel(&sv, &dv, r.dx, r.dy, r.ksize, r.scale, r.border, st);
        case IPFC_OP_MEDIAN: return ipfc_median_blur(&sv, &dv, r.ksize, r.border, st);
        case IPFC_OP_FILTER2D:
            return ipfc_filter2d(&sv, &dv, q.taps.data(), r.kw, r.kh, -1, -1, r.border, r.delta, r.border_value, st);
        case IPFC_OP_BOX: return ipfc_box_filter(&sv, &dv, r.ksize, r.ksize, 1, r.border, r.border_value, st);
        case IPFC_OP_ERODE:
        case IPFC_OP_DILATE: {
            std::vector<uint8_t> se((size_t)r.ksize * r.ksize, 1);
            return r.op == IPFC_OP_ERODE ? ipfc_erode(&sv, &dv, se.data(), r.ksize, r.ksize, 1, st)
                                         : ipfc_dilate(&sv, &dv, se.data(), r.ksize, r.ksize, 1, st);
        }
        default: return set_error(IPFC_ERR_INVALID, "ipf: server: unknown op %d", r.op);
    }
}

// Enqueues one group on one stream; the group's requests carry their
// status (a failed request still completes, with its error code).
void dispatch_group(ipfc_server* s, Group& g, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    // device buffers and input copies
    auto pool_alloc = [&](void** p, size_t bytes) -> cudaError_t {
        const long long nth = s->fail_alloc_nth.load();
        if (nth > 0 && ++s->allocs == nth) return cudaErrorMemoryAllocation;  // injected (host side)
        return cudaMallocFromPoolAsync(p, bytes, s->pool, st);
    };
    for (Req& q : g.reqs) {
        const ipfc_request& r = q.r;
        if (r.src.mem == IPFC_MEM_HOST) {
            q.dspitch = row_bytes_of(r.src);
            e = pool_alloc(&q.dsrc, round256((size_t)q.dspitch * r.src.height));
            if (e == cudaSuccess)
                e = cudaMemcpy2DAsync(q.dsrc, (size_t)q.dspitch, r.src.data, (size_t)pitch_of_img(r.src),
                                      (size_t)q.dspitch, (size_t)r.src.height, cudaMemcpyHostToDevice, st);
        } else {
            q.dsrc = r.src.data;
            q.dspitch = pitch_of_img(r.src);
        }
        if (e == cudaSuccess && r.dst.mem == IPFC_MEM_HOST) {
            q.ddpitch = row_bytes_of(r.dst);
            e = pool_alloc(&q.ddst, round256((size_t)q.ddpitch * r.dst.height));
        } else if (e == cudaSuccess) {
            q.ddst = r.dst.data;
            q.ddpitch = pitch_of_img(r.dst);
        }
        if (e != cudaSuccess) q.status = cuda_status(e, "server");
        e = cudaSuccess;
    }
    // kernels: the batchable requests as one batch plan (separable group
    // launches and persistent queue kernels)
    std::vector<HostItem> items;
    std::vector<TuneVal> vals;
    std::vector<int> idx;
    if (s->cfg.batch) {
        for (size_t i = 0; i < g.reqs.size(); ++i) {
            Req& q = g.reqs[i];
            if (q.status != IPFC_OK || !batchable(q.r)) continue;
            HostItem h;
            if (!batch_item(q, &h)) continue;
            items.push_back(h);
            vals.push_back(tuned_or_default(h.it.kind, h.it.K, h.it.C, h.W, h.H));
            idx.push_back((int)i);
        }
    }
    std::vector<char> done(g.reqs.size(), 0);
    if (items.size() >= 2) {
        HostPlan p;
        build_host_plan(items, vals, &p);
        int grid[kBatchClasses];
        e = plan_grids(p, grid);
        void* dplan = nullptr;
        const size_t ib = round256(sizeof(BatchItem) * p.items.size());
        const size_t tb = round256(sizeof(BatchTile) * p.tiles.size());
        if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&dplan, ib + tb + 256, s->pool, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dplan, p.items.data(), sizeof(BatchItem) * p.items.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync((char*)dplan + ib, p.tiles.data(), sizeof(BatchTile) * p.tiles.size(),
                                cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = launch_plan((const BatchItem*)dplan, (const BatchTile*)((char*)dplan + ib),
                            (unsigned*)((char*)dplan + ib + tb), p, grid, st, nullptr, 0, nullptr, nullptr);
        if (dplan) cudaFreeAsync(dplan, st);
        for (int i : idx) {
            done[i] = 1;
            if (e != cudaSuccess) g.reqs[i].status = cuda_status(e, "server (batch)");
        }
        if (e == cudaSuccess) {
            s->st_batch_launches++;
            s->st_batched += (long long)idx.size();
        }
        e = cudaSuccess;
    }
    for (size_t i = 0; i < g.reqs.size(); ++i) {
        Req& q = g.reqs[i];
        if (done[i] || q.status != IPFC_OK) continue;
        const int rc = run_single(q, st);
        if (rc != IPFC_OK) q.status = rc;
    }
    // results back, memory returned to the pool in stream order
    for (Req& q : g.reqs) {
        const ipfc_request& r = q.r;
        if (r.dst.mem == IPFC_MEM_HOST && q.ddst) {
            if (q.status == IPFC_OK) {
                e = cudaMemcpy2DAsync(r.dst.data, (size_t)pitch_of_img(r.dst), q.ddst, (size_t)q.ddpitch,
                                      (size_t)q.ddpitch, (size_t)r.dst.height, cudaMemcpyDeviceToHost, st);
                if (e != cudaSuccess) q.status = cuda_status(e, "server");
            }
            cudaFreeAsync(q.ddst, st);
        }
        if (r.src.mem == IPFC_MEM_HOST && q.dsrc) cudaFreeAsync(q.dsrc, st);
    }
    e = cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(g.done, st);
    if (e != cudaSuccess) {
        cudaStreamSynchronize(st);
        if (g.done) cudaEventDestroy(g.done);
        g.done = nullptr;
    }
    s->st_groups++;
}

void scheduler(ipfc_server* s) {
    cudaSetDevice(s->device);
    for (;;) {
        bool progressed = false;
        // 1. completions
        for (size_t i = 0; i < s->inflight.size();) {
            Group& g = s->inflight[i];
            const cudaError_t q = g.done ? cudaEventQuery(g.done) : cudaSuccess;
            if (q == cudaErrorNotReady) {
                ++i;
                continue;
            }
            if (q != cudaSuccess)
                for (Req& r : g.reqs) r.status = cuda_status(q, "server");
            if (g.done) cudaEventDestroy(g.done);
            complete_group(s, g);
            s->inflight.erase(s->inflight.begin() + (long)i);
            progressed = true;
        }
        // 2. admission
        std::vector<Req> admitted;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stop && s->pending.empty() && s->inflight.empty()) break;
            const double t = s->now();
            while (!s->pending.empty()) {
                Req& q = s->pending.front();
                if (q.arrival > t) break;
                if (q.dev_bytes > s->cfg.device_budget_bytes) {  // can never fit
                    ipfc_completion c{q.ticket, IPFC_ERR_NOMEM, q.arrival, t, t};
                    s->completions.push_back(c);
                    s->finished++;
                    s->st_failed++;
                    s->pending.pop_front();
                    s->cv_done.notify_all();
                    continue;
                }
                if (s->used_slots >= s->cfg.max_inflight || s->used_bytes + q.dev_bytes > s->cfg.device_budget_bytes)
                    break;
                s->used_slots++;
                s->used_bytes += q.dev_bytes;
                q.admitted = t;
                admitted.push_back(std::move(q));
                s->pending.pop_front();
            }
            s->st_max_slots = std::max<long long>(s->st_max_slots.load(), s->used_slots);
            s->st_max_bytes = std::max<long long>(s->st_max_bytes.load(), (long long)s->used_bytes);
            if (admitted.empty() && s->inflight.empty() && !progressed) {
                // idle: sleep until a submission or the next arrival is due
                if (s->pending.empty()) {
                    s->cv_submit.wait_for(lk, std::chrono::milliseconds(50));
                } else {
                    const double wait = s->pending.front().arrival - s->now();
                    if (wait > 0) s->cv_submit.wait_for(lk, std::chrono::duration<double>(std::min(wait, 0.05)));
                }
                continue;
            }
        }
        // 3. dispatch: round-robin over the streams
        if (!admitted.empty()) {
            const int ns = (int)s->streams.size();
            std::vector<Group> groups((size_t)ns);
            for (size_t i = 0; i < admitted.size(); ++i)
                groups[(s->next_stream + i) % ns].reqs.push_back(std::move(admitted[i]));
            s->next_stream = (int)((s->next_stream + admitted.size()) % ns);
            for (int k = 0; k < ns; ++k) {
                if (groups[k].reqs.empty()) continue;
                dispatch_group(s, groups[k], s->streams[k]);
                s->inflight.push_back(std::move(groups[k]));
            }
        } else if (!progressed) {
            std::this_thread::yield();
        }
    }
}

}  // namespace

extern "C" {

int ipfc_server_fail_allocation(ipfc_server* s, long long nth) {
    if (!s || nth < 0) return set_error(IPFC_ERR_INVALID, "ipf: server: invalid argument");
    s->fail_alloc_nth.store(nth);
    return IPFC_OK;
}

int ipfc_server_create(ipfc_server** out, const ipfc_server_config* cfg) {
    if (!out) return set_error(IPFC_ERR_INVALID, "ipf: server: null output pointer");
    ipfc_server_config c;
    c.device_budget_bytes = (size_t)40 << 30;
    c.max_inflight = 64;
    c.streams = 4;
    c.batch = 1;
    if (cfg) c = *cfg;
    if (c.max_inflight < 1 || c.streams < 1 || c.streams > 64 || c.device_budget_bytes == 0)
        return set_error(IPFC_ERR_INVALID, "ipf: server: invalid configuration");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, "server");
    ipfc_server* s = new ipfc_server();
    s->cfg = c;
    s->device = dev;
    s->epoch = Clock::now();
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    e = cudaMemPoolCreate(&s->pool, &props);
    if (e == cudaSuccess) {
        unsigned long long thr = (unsigned long long)c.device_budget_bytes;
        e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    for (int i = 0; i < c.streams && e == cudaSuccess; ++i) {
        cudaStream_t st = nullptr;
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e == cudaSuccess) s->streams.push_back(st);
    }
    if (e != cudaSuccess) {
        for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
        if (s->pool) cudaMemPoolDestroy(s->pool);
        delete s;
        return cuda_status(e, "server");
    }
    s->worker = std::thread(scheduler, s);
    *out = s;
    return IPFC_OK;
}

int ipfc_server_destroy(ipfc_server* s) {
    if (!s) return IPFC_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_submit.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (cudaStream_t st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return IPFC_OK;
}

double ipfc_server_now(const ipfc_server* s) { return s ? s->now() : 0.0; }

int ipfc_server_submit(ipfc_server* s, const ipfc_request* r, unsigned long long* ticket) {
    if (!s || !r) return set_error(IPFC_ERR_INVALID, "ipf: server: null argument");
    if (r->op < IPFC_OP_GAUSSIAN || r->op > IPFC_OP_DILATE)
        return set_error(IPFC_ERR_INVALID, "ipf: server: unknown op %d", r->op);
    const ipfc_image& a = r->src;
    const ipfc_image& b = r->dst;
    if (!a.data || !b.data || a.width <= 0 || a.height <= 0 || a.channels < 1)
        return set_error(IPFC_ERR_INVALID, "ipf: server: requests need non-empty images");
    if (b.width != a.width || b.height != a.height || b.channels != a.channels)
        return set_error(IPFC_ERR_INVALID, "ipf: server: destination shape does not match source");
    if ((a.mem != IPFC_MEM_HOST && a.mem != IPFC_MEM_DEVICE) || (b.mem != IPFC_MEM_HOST && b.mem != IPFC_MEM_DEVICE))
        return set_error(IPFC_ERR_INVALID, "ipf: server: invalid memory kind");
    if (a.dtype < IPFC_U8 || a.dtype > IPFC_F64 || b.dtype < IPFC_U8 || b.dtype > IPFC_F64)
        return set_error(IPFC_ERR_INVALID, "ipf: server: invalid element type");
    if (r->op == IPFC_OP_FILTER2D && (!r->kernel || r->kw <= 0 || r->kh <= 0))
        return set_error(IPFC_ERR_INVALID, "ipf: filter2D: kernel must be a non-empty single-channel image");
    Req q;
    q.r = *r;
    if (r->op == IPFC_OP_FILTER2D) q.taps.assign(r->kernel, r->kernel + (size_t)r->kw * r->kh);
    q.dev_bytes = request_bytes(*r);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return set_error(IPFC_ERR_INVALID, "ipf: server: stopped");
        q.ticket = s->next_ticket++;
        q.arrival = r->arrival >= 0 ? r->arrival : s->now();
        if (ticket) *ticket = q.ticket;
        // arrival order: requests with explicit times may come out of order
        auto pos = s->pending.end();
        while (pos != s->pending.begin() && (pos - 1)->arrival > q.arrival) --pos;
        s->pending.insert(pos, std::move(q));
        s->submitted++;
    }
    s->cv_submit.notify_all();
    return IPFC_OK;
}

int ipfc_server_poll(ipfc_server* s, ipfc_completion* out, int max, int* n, int wait_ms) {
    if (!s || !n || (max > 0 && !out)) return set_error(IPFC_ERR_INVALID, "ipf: server: null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->completions.empty() && wait_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->completions.empty(); });
    int k = 0;
    while (k < max && !s->completions.empty()) {
        out[k++] = s->completions.front();
        s->completions.pop_front();
    }
    *n = k;
    return IPFC_OK;
}

int ipfc_server_drain(ipfc_server* s, int timeout_ms) {
    if (!s) return set_error(IPFC_ERR_INVALID, "ipf: server: null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms < 0 ? 1 << 30 : timeout_ms),
                                        [&] { return s->finished == s->submitted; });
    return ok ? IPFC_OK : set_error(IPFC_ERR_TIMEOUT, "ipf: server: drain timed out");
}

int ipfc_server_stats(const ipfc_server* s, int what, double* v) {
    if (!s || !v) return set_error(IPFC_ERR_INVALID, "ipf: server: null argument");
    switch (what) {
        case IPFC_SERVER_STAT_GROUPS: *v = (double)s->st_groups.load(); break;
        case IPFC_SERVER_STAT_BATCHED: *v = (double)s->st_batched.load(); break;
        case IPFC_SERVER_STAT_BATCH_LAUNCHES: *v = (double)s->st_batch_launches.load(); break;
        case IPFC_SERVER_STAT_MAX_INFLIGHT: *v = (double)s->st_max_slots.load(); break;
        case IPFC_SERVER_STAT_MAX_BYTES: *v = (double)s->st_max_bytes.load(); break;
        case IPFC_SERVER_STAT_FAILED: *v = (double)s->st_failed.load(); break;
        default: return set_error(IPFC_ERR_INVALID, "ipf: server: unknown statistic %d", what);
    }
    return IPFC_OK;
}

}  // extern "C"
