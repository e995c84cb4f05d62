// Native serving core: power-flow and N-1 requests over several plans, continuously batched
// on one GPU.  Built on the public C ABI (pf_n1_prepare, pf_batch_device_scratch).
//
// Every grid keeps its plan, base-case voltages and injections and its branch-removal
// coefficients; device memory is one arena of the HBM budget, carved first-fit into one region
// per admitted request (inputs, outputs and the kernel's working memory), so serving allocates
// no device memory after creation.  Requests are admitted oldest first when a stream slot is
// free and their region fits; each runs as its own launch on its slot's stream with pinned
// staging, so requests that arrive while others run overlap with them on the device.  Results
// are copied into the caller's buffers when the slot's event has completed.
#include "../../include/lightsim2grid_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <complex>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pf_capi_internal.hpp"

namespace {

using cplx = std::complex<double>;

int fail(const std::string &msg) {
    l2g::set_last_error(msg);
    return -1;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// the latency split keeps at most this many requests per grid and kind between resets
constexpr size_t kSplitCap = size_t(1) << 18;

// host clock for the latency split (seconds)
double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// First-fit allocator over [0, size): holes sorted by offset, coalesced on release.
struct Arena {
    size_t size = 0;
    std::list<std::pair<size_t, size_t>> holes;
    void init(size_t s) {
        size = s;
        holes.assign(1, {0, s});
    }
    bool alloc(size_t n, size_t &off) {
        n = align256(n);
        for (auto it = holes.begin(); it != holes.end(); ++it)
            if (it->second >= n) {
                off = it->first;
                if (it->second == n) holes.erase(it);
                else {
                    it->first += n;
                    it->second -= n;
                }
                return true;
            }
        return false;
    }
    void release(size_t off, size_t n) {
        n = align256(n);
        auto it = holes.begin();
        while (it != holes.end() && it->first < off) ++it;
        it = holes.insert(it, {off, n});
        auto nx = std::next(it);
        if (nx != holes.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            holes.erase(nx);
        }
        if (it != holes.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                holes.erase(it);
            }
        }
    }
};

struct Grid {
    pf_plan *plan = nullptr;
    int n = 0, nbr = 0, ctas = 0, ctas_per_sm = 1;
    int cls = -1;  // device loop: its class
    std::vector<cplx> S;            // base injections (host)
    void *dV0 = nullptr, *dS = nullptr;
    std::vector<int> cptr, rows, cols;
    std::vector<cplx> vals;
    double tol = 1e-8;
    int max_iter = 10;
};

struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    unsigned char *pin_in = nullptr, *pin_out = nullptr;
    unsigned char *pin_out_dev = nullptr;  // device address of pin_out
    bool high = false;  // on a high-priority stream
};

// Requests with at most this many instance-buses run on high-priority streams: the block
// scheduler then dispatches their CTAs before the pending CTAs of large batches launched
// earlier, so a small request does not wait behind them.
constexpr long long kSmallWork = 20000;
// ... and whose grid has at most this many buses: one instance of a larger grid keeps its SM for a
// millisecond or more (the whole shared memory of the 2,848-bus mixed plan), so it counts as large
// for the SM reservation below even alone
constexpr int kHeavyBuses = 2000;

// Priorities reorder pending CTAs only: a CTA of a large batch that is already resident keeps its
// SM until its instance is solved (milliseconds on the largest grids).  So large requests are
// also admitted only while the SMs their CTAs occupy, summed over the large requests in flight,
// stay within num_sms - reserved_sms: the reserved SMs are left to small requests.

struct Req {
    long long id = 0;
    int grid = 0, kind = 0, ncases = 0, ninst = 0;
    std::vector<double> scale;
    std::vector<int> solv;                 // N-1: per case, solvable
    std::vector<int> optr, opos;
    std::vector<cplx> oval;
    double *V = nullptr;                   // caller buffers, case order
    int *iters = nullptr, *errs = nullptr;
    size_t scratch = 0, outs = 0, ins = 0, bytes = 0, off = 0;
    int slot = -1;
    bool small = true;   // instance-buses <= kSmallWork on a grid of at most kHeavyBuses buses
    int ctas = 0;        // CTAs of its launch
    int sms = 0;         // SMs those CTAs occupy (large requests)
    int cls = -1;        // device loop: the loop class that runs it
    bool slot_freed = false;  // delivered by the polling thread, slot already returned
    double t_sub = 0.0, t_adm = 0.0;  // host clock at submission and at admission (launch or publish)
};

// Device-resident request loop: the grids whose plans share an LU placement form a class, served by
// one persistent launch of the Newton kernel in queue mode.  The host appends each admitted
// request's segment and jobs to the class's rings in device memory through copies on a feeder
// stream, then advances the ring's tail the same way (stream order: the entries land before the
// tail); the kernel's CTAs claim jobs as they are published, write the results into the slot's
// mapped pinned staging and count the finished instances per slot in mapped host memory.  After
// kIdlePolls empty polls a CTA closes the loop (all its CTAs leave once the ring is empty); the host
// closes it the same way when it switches modes or is destroyed, and launches it again whenever
// work is published while it is not running.
constexpr int kIdlePolls = 2000000;  // ~1-2 s of empty polls (500 ns naps) before a loop closes

struct LoopClass {
    std::vector<int> grids;
    l2g::LoopShape sh;
    int ctas = 0;
    unsigned char *scratch = nullptr;   // device: per-CTA slabs
    l2g::QueueJob *jobs = nullptr;      // device: job ring
    int cap = 0;
    l2g::Segment *segs = nullptr;       // device: one segment per slot
    int *head = nullptr, *tail = nullptr, *closing = nullptr;  // device
    l2g::QueueJob *job_stage = nullptr; // pinned: the ring's host image
    l2g::Segment *seg_stage = nullptr;  // pinned: one segment per slot
    int *tail_stage = nullptr;          // pinned: a ring of published tail values
    int ntail = 0, tail_next = 0;
    int published = 0;                  // jobs published
    cudaStream_t kst = nullptr, fst = nullptr;
    cudaEvent_t kev = nullptr;
    bool launched = false;
    int inflight = 0;                   // its requests not yet complete
};

}  // namespace

struct pf_server {
    std::vector<Grid> grids;
    int max_k = 64, nslots = 0;
    size_t budget = 0, in_use = 0, in_cap = 0, out_cap = 0;
    unsigned char *arena_ptr = nullptr;
    Arena arena;
    std::vector<Slot> slots;
    std::vector<int> free_high, free_low;
    int *djf = nullptr, *djc = nullptr;
    std::deque<Req *> pending;
    std::vector<Req *> inflight;
    // SM reservation for small requests (see kSmallWork)
    int num_sms = 1, reserved_sms = 0, large_ctas = 1 << 30, large_sms_inflight = 0;
    // delivery: copying a finished large request's rows from pinned staging into the caller's
    // arrays (megabytes for N-1 batches of the large grids) runs on worker threads, so the polling
    // thread keeps admitting and completing other requests meanwhile; small requests' rows are
    // copied by the polling thread itself and returned by the same poll
    std::vector<std::thread> workers;
    mutable std::mutex mu;
    std::condition_variable cv;
    std::deque<Req *> to_deliver;   // device work done, rows not yet copied
    std::vector<Req *> delivered;   // rows copied: slot (unless freed) and id returned by the next poll
    bool stop = false;
    // device-resident request loop (pf_server_device_loop)
    bool loop = false;
    std::vector<LoopClass> classes;
    int *done_host = nullptr, *done_dev = nullptr;  // mapped: instances finished per slot
    int req_seq = 0;
    // latency split per grid and kind (index 2 * grid + kind): admission wait (submission to
    // launch or publication) and device time (that to the poll that saw it finished), ms
    std::vector<std::vector<float>> wait_ms, run_ms;
};

namespace {

void stop_workers(pf_server *s) {
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    for (std::thread &t : s->workers)
        if (t.joinable()) t.join();
    s->workers.clear();
}

void free_loop(pf_server *s) {
    for (LoopClass &c : s->classes) {
        // close the loop (its CTAs leave once the ring is empty) and wait for it
        if (c.closing && c.fst) {
            cudaMemsetAsync(c.closing, 0xff, sizeof(int), c.fst);
            cudaStreamSynchronize(c.fst);
        }
        if (c.kst) cudaStreamSynchronize(c.kst);
        if (c.fst) cudaStreamSynchronize(c.fst);
        for (void *p : {(void *)c.scratch, (void *)c.jobs, (void *)c.segs, (void *)c.head})
            if (p) cudaFree(p);
        for (void *p : {(void *)c.job_stage, (void *)c.seg_stage, (void *)c.tail_stage})
            if (p) cudaFreeHost(p);
        if (c.kev) cudaEventDestroy(c.kev);
        if (c.kst) cudaStreamDestroy(c.kst);
        if (c.fst) cudaStreamDestroy(c.fst);
    }
    s->classes.clear();
    if (s->done_host) cudaFreeHost(s->done_host);
    s->done_host = s->done_dev = nullptr;
    s->loop = false;
}

void destroy(pf_server *s) {
    stop_workers(s);
    free_loop(s);
    for (Req *r : s->to_deliver) delete r;
    for (Req *r : s->delivered) delete r;
    for (Grid &g : s->grids) {
        if (g.dV0) cudaFree(g.dV0);
        if (g.dS) cudaFree(g.dS);
    }
    for (Slot &sl : s->slots) {
        if (sl.ev) cudaEventDestroy(sl.ev);
        if (sl.st) cudaStreamDestroy(sl.st);
        if (sl.pin_in) cudaFreeHost(sl.pin_in);
        if (sl.pin_out) cudaFreeHost(sl.pin_out);
    }
    if (s->arena_ptr) cudaFree(s->arena_ptr);
    if (s->djf) cudaFree(s->djf);
    if (s->djc) cudaFree(s->djc);
    for (Req *r : s->pending) delete r;
    for (Req *r : s->inflight) delete r;
    delete s;
}

// Inputs of a request: the scaled injections (PF) or its overrides; sizes of its region.
int prepare(pf_server *s, Req *r) {
    Grid &g = s->grids[r->grid];
    if (r->kind == 0) {
        r->ninst = 1;
        r->ins = align256((size_t)g.n * 16);
    } else {
        std::vector<int> cp(r->ncases + 1, 0), rows, cols;
        std::vector<cplx> vals;
        for (int c = 0; c < r->ncases; ++c) {
            const int b = r->solv[c];  // branch id, replaced by the solvable flag below
            if (b < 0 || b >= g.nbr) return fail("pf_server_submit: branch id out of range");
            for (int q = g.cptr[b]; q < g.cptr[b + 1]; ++q) {
                rows.push_back(g.rows[q]);
                cols.push_back(g.cols[q]);
                vals.push_back(g.vals[q]);
            }
            cp[c + 1] = (int)rows.size();
        }
        if (rows.empty()) {
            rows.push_back(0);
            cols.push_back(0);
            vals.push_back(0.0);
        }
        const int cap = std::max(cp[r->ncases], 1);
        r->optr.assign(r->ncases + 1, 0);
        r->opos.assign(cap, 0);
        r->oval.assign(cap, 0.0);
        std::vector<int> solv(r->ncases, 0);
        const int w = pf_n1_prepare(g.plan, r->ncases, cp.data(), rows.data(), cols.data(),
                                    reinterpret_cast<const double *>(vals.data()), solv.data(), r->optr.data(),
                                    r->opos.data(), reinterpret_cast<double *>(r->oval.data()), cap);
        if (w < 0) return w;
        r->solv = solv;
        r->ninst = 0;
        for (int c = 0; c < r->ncases; ++c) r->ninst += solv[c];
        r->optr.resize(r->ninst + 1);
        r->opos.resize(std::max(w, 1));
        r->oval.resize(std::max(w, 1));
        r->ins = align256((size_t)(r->ninst + 1) * 4) + align256(r->opos.size() * 4) + align256(r->oval.size() * 16);
    }
    if (r->ninst > s->max_k) return fail("pf_server_submit: request has more instances than the server's maximum");
    if (r->ins > s->in_cap) return fail("pf_server_submit: request inputs exceed the staging buffers");
    r->small = (long long)r->ninst * g.n <= kSmallWork && g.n <= kHeavyBuses;
    int ctas = std::max(1, std::min(r->ninst, g.ctas));
    if (!r->small) ctas = std::max(1, std::min(ctas, s->large_ctas));
    r->ctas = ctas;
    r->sms = (ctas + g.ctas_per_sm - 1) / g.ctas_per_sm;
    // device loop: the small requests of grids that a loop serves go through it (their CTAs are
    // resident); the others are launched as usual
    r->cls = (s->loop && r->small) ? g.cls : -1;
    r->scratch = (r->ninst && r->cls < 0) ? align256((size_t)pf_scratch_bytes(g.plan, ctas)) : 0;
    r->outs = 0;  // the kernel writes the results straight into the slot's mapped pinned staging
    r->bytes = r->scratch + r->outs + r->ins;
    return 0;
}

int launch(pf_server *s, Req *r) {
    Grid &g = s->grids[r->grid];
    Slot &sl = s->slots[r->slot];
    unsigned char *base = s->arena_ptr + r->off;
    unsigned char *scr = base, *in = base + r->scratch + r->outs;
    // outputs: the slot's pinned staging, mapped into the device address space (the kernel writes
    // each instance's row there as it finishes: no copy engine in the way of other requests)
    unsigned char *out = sl.pin_out_dev;
    cudaError_t e = cudaSuccess;
    if (r->ninst > 0) {
        pf_device_batch b{};
        b.n_inst = r->ninst;
        b.V0 = g.dV0;
        b.max_iter = g.max_iter;
        b.tol = g.tol;
        b.job_first = s->djf;
        b.job_count = s->djc;
        b.njobs = r->ninst;
        b.Vout = out;
        b.iters = reinterpret_cast<int *>(out + (size_t)r->ninst * g.n * 16);
        b.errs = b.iters + r->ninst;
        if (r->kind == 0) {
            cplx *S = reinterpret_cast<cplx *>(sl.pin_in);
            for (int i = 0; i < g.n; ++i) S[i] = g.S[i] * r->scale[i];
            e = cudaMemcpyAsync(in, sl.pin_in, (size_t)g.n * 16, cudaMemcpyHostToDevice, sl.st);
            b.Sbus = in;
        } else {
            const size_t a1 = align256((size_t)(r->ninst + 1) * 4), a2 = align256(r->opos.size() * 4);
            std::memcpy(sl.pin_in, r->optr.data(), (size_t)(r->ninst + 1) * 4);
            std::memcpy(sl.pin_in + a1, r->opos.data(), r->opos.size() * 4);
            std::memcpy(sl.pin_in + a1 + a2, r->oval.data(), r->oval.size() * 16);
            e = cudaMemcpyAsync(in, sl.pin_in, a1 + a2 + r->oval.size() * 16, cudaMemcpyHostToDevice, sl.st);
            b.Sbus = g.dS;
            b.ovr_ptr = reinterpret_cast<const int *>(in);
            b.ovr_pos = reinterpret_cast<const int *>(in + a1);
            b.ovr_val = in + a1 + a2;
        }
        if (e != cudaSuccess) return fail(std::string("pf_server: upload: ") + cudaGetErrorString(e));
        const int rc = pf_batch_device_scratch(g.plan, &b, scr, (long long)r->scratch, sl.st);
        if (rc != 0) return rc;
    }
    e = cudaEventRecord(sl.ev, sl.st);
    if (e != cudaSuccess) return fail(std::string("pf_server: event: ") + cudaGetErrorString(e));
    return 0;
}

// Device loop: the request's inputs, segment and jobs go to the class's rings on the feeder stream,
// then the new tail; the loop is launched when it is not running.
int publish(pf_server *s, Req *r) {
    Grid &g = s->grids[r->grid];
    Slot &sl = s->slots[r->slot];
    LoopClass &c = s->classes[r->cls];
    unsigned char *in = s->arena_ptr + r->off;
    unsigned char *out = sl.pin_out_dev;
    cudaError_t e = cudaSuccess;
    pf_device_batch b{};
    b.n_inst = r->ninst;
    b.V0 = g.dV0;
    b.max_iter = g.max_iter;
    b.tol = g.tol;
    b.Vout = out;
    b.iters = reinterpret_cast<int *>(out + (size_t)r->ninst * g.n * 16);
    b.errs = b.iters + r->ninst;
    if (r->kind == 0) {
        cplx *S = reinterpret_cast<cplx *>(sl.pin_in);
        for (int i = 0; i < g.n; ++i) S[i] = g.S[i] * r->scale[i];
        e = cudaMemcpyAsync(in, sl.pin_in, (size_t)g.n * 16, cudaMemcpyHostToDevice, c.fst);
        b.Sbus = in;
    } else {
        const size_t a1 = align256((size_t)(r->ninst + 1) * 4), a2 = align256(r->opos.size() * 4);
        std::memcpy(sl.pin_in, r->optr.data(), (size_t)(r->ninst + 1) * 4);
        std::memcpy(sl.pin_in + a1, r->opos.data(), r->opos.size() * 4);
        std::memcpy(sl.pin_in + a1 + a2, r->oval.data(), r->oval.size() * 16);
        e = cudaMemcpyAsync(in, sl.pin_in, a1 + a2 + r->oval.size() * 16, cudaMemcpyHostToDevice, c.fst);
        b.Sbus = g.dS;
        b.ovr_ptr = reinterpret_cast<const int *>(in);
        b.ovr_pos = reinterpret_cast<const int *>(in + a1);
        b.ovr_val = in + a1 + a2;
    }
    if (e != cudaSuccess) return fail(std::string("pf_server: upload: ") + cudaGetErrorString(e));
    l2g::Segment &sg = c.seg_stage[r->slot];
    int rc = l2g::loop_segment(g.plan, &b, c.sh, c.scratch, &sg);
    if (rc != 0) return rc;
    e = cudaMemcpyAsync(c.segs + r->slot, &sg, sizeof(l2g::Segment), cudaMemcpyHostToDevice, c.fst);
    if (e != cudaSuccess) return fail(std::string("pf_server: segment: ") + cudaGetErrorString(e));
    // the jobs: one per instance, in the ring (two copies when it wraps)
    const int seq = s->req_seq++;
    s->done_host[r->slot] = 0;  // read by the host only; the loop adds once it runs the jobs
    const int start = c.published % c.cap;
    for (int i = 0; i < r->ninst; ++i) c.job_stage[(start + i) % c.cap] = l2g::QueueJob{r->slot, i, 1, seq};
    const int first_len = std::min(r->ninst, c.cap - start);
    e = cudaMemcpyAsync(c.jobs + start, c.job_stage + start, (size_t)first_len * sizeof(l2g::QueueJob),
                        cudaMemcpyHostToDevice, c.fst);
    if (e == cudaSuccess && r->ninst > first_len)
        e = cudaMemcpyAsync(c.jobs, c.job_stage, (size_t)(r->ninst - first_len) * sizeof(l2g::QueueJob),
                            cudaMemcpyHostToDevice, c.fst);
    c.published += r->ninst;
    // the new tail, from a ring of pinned values (each stays untouched until its copy has run:
    // the ring is longer than the requests that can be in flight)
    int *tv = c.tail_stage + c.tail_next;
    c.tail_next = (c.tail_next + 1) % c.ntail;
    *tv = c.published;
    if (e == cudaSuccess) e = cudaMemcpyAsync(c.tail, tv, sizeof(int), cudaMemcpyHostToDevice, c.fst);
    if (e != cudaSuccess) return fail(std::string("pf_server: queue: ") + cudaGetErrorString(e));
    c.inflight += 1;
    if (!c.launched) {
        if ((e = cudaMemsetAsync(c.closing, 0, sizeof(int), c.kst)) != cudaSuccess)
            return fail(std::string("pf_server: loop reset: ") + cudaGetErrorString(e));
        rc = l2g::loop_launch(c.sh, sg,
                              l2g::DevQueue{c.jobs, c.cap, c.segs, c.head, c.tail, s->done_dev, c.closing, kIdlePolls},
                              c.ctas, c.kst);
        if (rc != 0) return rc;
        if ((e = cudaEventRecord(c.kev, c.kst)) != cudaSuccess)
            return fail(std::string("pf_server: loop event: ") + cudaGetErrorString(e));
        c.launched = true;
    }
    return 0;
}

// Results of a finished request into the caller's buffers, in case order.
void deliver(pf_server *s, Req *r) {
    Grid &g = s->grids[r->grid];
    const unsigned char *po = s->slots[r->slot].pin_out;
    const cplx *V = reinterpret_cast<const cplx *>(po);
    const int *it = reinterpret_cast<const int *>(po + (size_t)r->ninst * g.n * 16);
    const int *er = it + r->ninst;
    cplx *Vo = reinterpret_cast<cplx *>(r->V);
    const int rows = r->kind == 0 ? 1 : r->ncases;
    int k = 0;
    for (int c = 0; c < rows; ++c) {
        const bool solved = r->kind == 0 || r->solv[c];
        if (!solved) {
            std::fill(Vo + (size_t)c * g.n, Vo + (size_t)(c + 1) * g.n, cplx(0.0, 0.0));
            r->iters[c] = 0;
            r->errs[c] = 1;  // SingularMatrix: the outage islands the grid (skipped)
            continue;
        }
        if (er[k] == 0) std::memcpy(Vo + (size_t)c * g.n, V + (size_t)k * g.n, (size_t)g.n * 16);
        else std::fill(Vo + (size_t)c * g.n, Vo + (size_t)(c + 1) * g.n, cplx(0.0, 0.0));
        r->iters[c] = it[k];
        r->errs[c] = er[k];
        ++k;
    }
}

void delivery_worker(pf_server *s) {
    for (;;) {
        Req *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait(lk, [s] { return s->stop || !s->to_deliver.empty(); });
            if (s->to_deliver.empty()) return;  // stopping
            r = s->to_deliver.front();
            s->to_deliver.pop_front();
        }
        deliver(s, r);
        std::lock_guard<std::mutex> lk(s->mu);
        s->delivered.push_back(r);
    }
}

// percentile q (0..1) of v (sorted in place), nearest rank
double pct(std::vector<float> &v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const size_t k = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
    return v[k];
}

}  // namespace

extern "C" {

int pf_server_create(const pf_server_grid *grids, int ngrids, long long hbm_budget, int slots, int max_instances,
                     pf_server **out) {
    if (!out || !grids || ngrids <= 0 || hbm_budget <= 0 || slots <= 0 || max_instances <= 0)
        return fail("pf_server_create: invalid argument");
    *out = nullptr;
    pf_server *s = new pf_server();
    s->max_k = max_instances;
    s->budget = (size_t)hbm_budget;
    int nmax = 0;
    cudaError_t e;
    for (int i = 0; i < ngrids; ++i) {
        const pf_server_grid &gi = grids[i];
        pf_plan_info info;
        if (!gi.plan || pf_plan_info_get(gi.plan, &info) != 0 || !gi.V0_ri || !gi.Sbus_ri || gi.nbr < 0 ||
            (gi.nbr > 0 && (!gi.case_ptr || !gi.rows || !gi.cols || !gi.vals_ri))) {
            destroy(s);
            return fail("pf_server_create: invalid grid " + std::to_string(i));
        }
        Grid g;
        g.plan = gi.plan;
        g.n = info.n;
        g.ctas = info.grid;
        g.ctas_per_sm = std::max(1, info.ctas_per_sm);
        g.nbr = gi.nbr;
        g.max_iter = gi.max_iter > 0 ? gi.max_iter : 10;
        g.tol = gi.tol > 0 ? gi.tol : 1e-8;
        const cplx *S = reinterpret_cast<const cplx *>(gi.Sbus_ri);
        g.S.assign(S, S + g.n);
        g.cptr.assign(gi.case_ptr, gi.case_ptr + gi.nbr + 1);
        const int nc = gi.nbr > 0 ? gi.case_ptr[gi.nbr] : 0;
        g.rows.assign(gi.rows, gi.rows + nc);
        g.cols.assign(gi.cols, gi.cols + nc);
        const cplx *cv = reinterpret_cast<const cplx *>(gi.vals_ri);
        g.vals.assign(cv, cv + nc);
        if ((e = cudaMalloc(&g.dV0, (size_t)g.n * 16)) != cudaSuccess ||
            (e = cudaMalloc(&g.dS, (size_t)g.n * 16)) != cudaSuccess ||
            (e = cudaMemcpy(g.dV0, gi.V0_ri, (size_t)g.n * 16, cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(g.dS, gi.Sbus_ri, (size_t)g.n * 16, cudaMemcpyHostToDevice)) != cudaSuccess) {
            s->grids.push_back(g);
            destroy(s);
            return fail(std::string("pf_server_create: grid upload: ") + cudaGetErrorString(e));
        }
        nmax = std::max(nmax, g.n);
        s->grids.push_back(g);
    }
    s->in_cap = std::max(align256((size_t)nmax * 16), (size_t)s->max_k * 40 * 24 + 1024);
    s->out_cap = (size_t)s->max_k * nmax * 16 + 8 * (size_t)s->max_k + 256;
    std::vector<int> jf(s->max_k), jc(s->max_k, 1);
    for (int i = 0; i < s->max_k; ++i) jf[i] = i;
    if ((e = cudaMalloc(&s->arena_ptr, s->budget)) != cudaSuccess ||
        (e = cudaMalloc(&s->djf, (size_t)s->max_k * 4)) != cudaSuccess ||
        (e = cudaMalloc(&s->djc, (size_t)s->max_k * 4)) != cudaSuccess ||
        (e = cudaMemcpy(s->djf, jf.data(), jf.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(s->djc, jc.data(), jc.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess) {
        destroy(s);
        return fail(std::string("pf_server_create: device memory: ") + cudaGetErrorString(e));
    }
    s->arena.init(s->budget);
    s->wait_ms.assign(2 * s->grids.size(), {});
    s->run_ms.assign(2 * s->grids.size(), {});
    s->slots.resize(slots);
    int prio_low = 0, prio_high = 0;
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    for (int i = 0; i < slots; ++i) {
        Slot &sl = s->slots[i];
        sl.high = i < (slots + 1) / 2;
        if ((e = cudaStreamCreateWithPriority(&sl.st, cudaStreamNonBlocking, sl.high ? prio_high : prio_low)) !=
                cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaHostAlloc(reinterpret_cast<void **>(&sl.pin_in), s->in_cap, cudaHostAllocDefault)) != cudaSuccess ||
            (e = cudaHostAlloc(reinterpret_cast<void **>(&sl.pin_out), s->out_cap, cudaHostAllocMapped)) !=
                cudaSuccess ||
            (e = cudaHostGetDevicePointer(reinterpret_cast<void **>(&sl.pin_out_dev), sl.pin_out, 0)) !=
                cudaSuccess) {
            destroy(s);
            return fail(std::string("pf_server_create: slots: ") + cudaGetErrorString(e));
        }
    }
    for (int i = slots - 1; i >= 0; --i) (s->slots[i].high ? s->free_high : s->free_low).push_back(i);
    s->nslots = slots;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, dev);
    s->num_sms = std::max(1, s->num_sms);
    s->reserved_sms = s->num_sms / 8;
    const unsigned hw = std::thread::hardware_concurrency();
    const int nworkers = (int)std::max(1u, std::min(4u, hw > 2 ? hw / 2 : 1u));
    try {
        for (int i = 0; i < nworkers; ++i) s->workers.emplace_back(delivery_worker, s);
    } catch (const std::exception &ex) {
        destroy(s);
        return fail(std::string("pf_server_create: delivery threads: ") + ex.what());
    }
    *out = s;
    return 0;
}

int pf_server_submit(pf_server *s, long long id, int grid, int kind, const double *scale, int nbranches,
                     const int *branches, double *V_out, int *iters_out, int *errs_out) {
    if (!s || grid < 0 || grid >= (int)s->grids.size() || (kind != 0 && kind != 1) || !V_out || !iters_out ||
        !errs_out || (kind == 0 && !scale) || (kind == 1 && (nbranches <= 0 || !branches)))
        return fail("pf_server_submit: invalid argument");
    Req *r = new Req();
    r->t_sub = now_s();
    r->id = id;
    r->grid = grid;
    r->kind = kind;
    r->V = V_out;
    r->iters = iters_out;
    r->errs = errs_out;
    if (kind == 0) {
        r->scale.assign(scale, scale + s->grids[grid].n);
    } else {
        r->ncases = nbranches;
        r->solv.assign(branches, branches + nbranches);
    }
    const int rc = prepare(s, r);
    if (rc != 0) {
        delete r;
        return rc;
    }
    if (r->bytes > s->budget) {
        delete r;
        return fail("pf_server_submit: the request needs more device memory than the whole budget");
    }
    s->pending.push_back(r);
    return 0;
}

int pf_server_poll(pf_server *s, long long *done_ids, int cap) {
    if (!s || (cap > 0 && !done_ids)) return fail("pf_server_poll: invalid argument");
    int nd = 0;
    // requests whose rows the workers copied: their slot is free again
    {
        std::lock_guard<std::mutex> lk(s->mu);
        size_t k = 0;
        for (; k < s->delivered.size() && nd < cap; ++k) {
            Req *r = s->delivered[k];
            if (!r->slot_freed) (s->slots[r->slot].high ? s->free_high : s->free_low).push_back(r->slot);
            done_ids[nd++] = r->id;
            delete r;
        }
        s->delivered.erase(s->delivered.begin(), s->delivered.begin() + (long)k);
    }
    // device completions: the device region is free; the rows go to a delivery worker (the slot's
    // pinned staging stays with the request until they are copied)
    bool queued = false;
    if (s->loop) std::atomic_thread_fence(std::memory_order_acquire);
    for (size_t i = 0; i < s->inflight.size();) {
        Req *r = s->inflight[i];
        if (r->cls >= 0) {
            // the loop counts the finished instances of the slot in mapped host memory
            const int d = *reinterpret_cast<volatile int *>(s->done_host + r->slot);
            if (d < r->ninst) {
                ++i;
                continue;
            }
            std::atomic_thread_fence(std::memory_order_acquire);
            if (r->ninst > 0) s->classes[r->cls].inflight -= 1;
        } else {
            const cudaError_t q = cudaEventQuery(s->slots[r->slot].ev);
            if (q == cudaErrorNotReady) {
                ++i;
                continue;
            }
            if (q != cudaSuccess) return fail(std::string("pf_server_poll: ") + cudaGetErrorString(q));
        }
        if (s->run_ms[2 * r->grid + r->kind].size() < kSplitCap) {
            const double t = now_s();
            s->wait_ms[2 * r->grid + r->kind].push_back((float)((r->t_adm - r->t_sub) * 1e3));
            s->run_ms[2 * r->grid + r->kind].push_back((float)((t - r->t_adm) * 1e3));
        }
        if (!r->small) s->large_sms_inflight -= r->sms;
        s->arena.release(r->off, r->bytes);
        s->in_use -= align256(r->bytes);
        s->inflight[i] = s->inflight.back();
        s->inflight.pop_back();
        if (r->small) {
            // a small request's rows (at most kSmallWork x 16 bytes) are copied here and its id
            // returned by this poll: handed to the workers it would wait behind the megabyte
            // copies of large N-1 results queued before it
            deliver(s, r);
            (s->slots[r->slot].high ? s->free_high : s->free_low).push_back(r->slot);
            if (nd < cap) {
                done_ids[nd++] = r->id;
                delete r;
            } else {
                // no room in the caller's array: the slot is free, the id comes with the next poll
                r->slot_freed = true;
                std::lock_guard<std::mutex> lk(s->mu);
                s->delivered.push_back(r);
            }
            continue;
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->to_deliver.push_back(r);
        }
        queued = true;
    }
    if (queued) s->cv.notify_all();
    // the loops: one that left (its CTAs ran out of published jobs) while requests of its class are
    // still open is launched again (their jobs are published and not yet claimed)
    for (LoopClass &c : s->classes) {
        if (!c.launched) continue;
        const cudaError_t q = cudaEventQuery(c.kev);
        if (q == cudaErrorNotReady) continue;
        if (q != cudaSuccess) return fail(std::string("pf_server_poll: request loop: ") + cudaGetErrorString(q));
        c.launched = false;
        if (c.inflight > 0) {
            cudaError_t e0 = cudaMemsetAsync(c.closing, 0, sizeof(int), c.kst);
            if (e0 != cudaSuccess) return fail(std::string("pf_server_poll: loop reset: ") + cudaGetErrorString(e0));
            const int rc = l2g::loop_launch(
                c.sh, c.seg_stage[0],
                l2g::DevQueue{c.jobs, c.cap, c.segs, c.head, c.tail, s->done_dev, c.closing, kIdlePolls}, c.ctas,
                c.kst);
            if (rc != 0) return rc;
            const cudaError_t e = cudaEventRecord(c.kev, c.kst);
            if (e != cudaSuccess) return fail(std::string("pf_server_poll: loop event: ") + cudaGetErrorString(e));
            c.launched = true;
        }
    }
    // admissions, oldest first; a large request that would take SMs from the reserve waits, and
    // the large ones behind it wait too (their order is kept), while small ones go past it
    const int large_budget = std::max(1, s->num_sms - s->reserved_sms);
    bool large_blocked = false;
    for (auto it = s->pending.begin();
         it != s->pending.end() && (!s->free_high.empty() || !s->free_low.empty());) {
        Req *r = *it;
        if (!r->small) {
            // a request needing more than the whole budget runs alone
            const bool fits = s->large_sms_inflight + r->sms <= large_budget || s->large_sms_inflight == 0;
            if (large_blocked || !fits) {
                large_blocked = true;
                ++it;
                continue;
            }
        }
        size_t off = 0;
        if (!s->arena.alloc(r->bytes, off)) break;
        it = s->pending.erase(it);
        if (!r->small) s->large_sms_inflight += r->sms;
        r->off = off;
        s->in_use += align256(r->bytes);
        // small requests prefer high-priority streams, large ones low-priority ones
        const bool small = r->small;
        std::vector<int> &pref = small ? s->free_high : s->free_low;
        std::vector<int> &other = small ? s->free_low : s->free_high;
        std::vector<int> &pool = pref.empty() ? other : pref;
        r->slot = pool.back();
        pool.pop_back();
        r->t_adm = now_s();
        int rc = 0;
        if (r->cls >= 0) {
            if (r->ninst > 0) rc = publish(s, r);
            else s->done_host[r->slot] = 0;  // every outage islanded: nothing to run
        } else {
            rc = launch(s, r);
        }
        s->inflight.push_back(r);
        if (rc != 0) return rc;
    }
    return nd;
}

int pf_server_device_loop(pf_server *s, int enable, int ctas_shared, int ctas_global) {
    if (!s || ctas_shared < 0 || ctas_global < 0) return fail("pf_server_device_loop: invalid argument");
    if (!s->pending.empty() || !s->inflight.empty())
        return fail("pf_server_device_loop: requests are queued or running; switch modes when idle");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->to_deliver.empty() || !s->delivered.empty())
            return fail("pf_server_device_loop: results are being delivered; switch modes when idle");
    }
    free_loop(s);
    if (!enable) return 0;
    // classes: the grids that have small requests (at most kHeavyBuses buses), split by LU
    // placement; the requests of larger grids keep their own launches, which spread over the SMs
    // the loops leave free
    std::vector<int> by[2];
    for (int i = 0; i < (int)s->grids.size(); ++i) {
        s->grids[i].cls = -1;
        pf_plan_info info;
        if (pf_plan_info_get(s->grids[i].plan, &info) != 0) return fail("pf_server_device_loop: plan info");
        if (s->grids[i].n <= kHeavyBuses) by[info.lu_in_shared ? 0 : 1].push_back(i);
    }
    if (by[0].empty() && by[1].empty()) return 0;  // nothing small to serve: launches only
    const int ncls = (!by[0].empty()) + (!by[1].empty());
    cudaError_t e = cudaSuccess;
    if ((e = cudaHostAlloc(reinterpret_cast<void **>(&s->done_host), sizeof(int) * (size_t)s->nslots,
                           cudaHostAllocMapped)) != cudaSuccess ||
        (e = cudaHostGetDevicePointer(reinterpret_cast<void **>(&s->done_dev), s->done_host, 0)) != cudaSuccess) {
        free_loop(s);
        return fail(std::string("pf_server_device_loop: completion counters: ") + cudaGetErrorString(e));
    }
    std::memset(s->done_host, 0, sizeof(int) * (size_t)s->nslots);
    s->classes.resize(ncls);
    int k = 0;
    for (int which = 0; which < 2; ++which) {
        if (by[which].empty()) continue;
        LoopClass &c = s->classes[k];
        c.grids = by[which];
        std::vector<pf_plan *> plans;
        for (int gi : c.grids) {
            plans.push_back(s->grids[gi].plan);
            s->grids[gi].cls = k;
        }
        int rc = l2g::loop_shape(plans.data(), (int)plans.size(), &c.sh);
        if (rc != 0) {
            free_loop(s);
            return rc;
        }
        // CTAs: a quarter of the SMs' worth for one class (the small requests' load; the rest of the
        // GPU stays with the launches of the large ones), an eighth each with two
        int want = which == 0 ? ctas_shared : ctas_global;
        if (want <= 0) want = std::max(1, (ncls == 1 ? s->num_sms / 4 : s->num_sms / 8) * c.sh.ctas_per_sm);
        c.ctas = std::min(want, s->num_sms * c.sh.ctas_per_sm);
        c.cap = 2 * s->nslots * s->max_k;
        c.ntail = 2 * s->nslots + 2;
        if ((e = cudaMalloc(&c.scratch, c.sh.slab * (size_t)c.ctas)) != cudaSuccess ||
            (e = cudaMalloc(&c.jobs, sizeof(l2g::QueueJob) * (size_t)c.cap)) != cudaSuccess ||
            (e = cudaMalloc(&c.segs, sizeof(l2g::Segment) * (size_t)s->nslots)) != cudaSuccess ||
            (e = cudaMalloc(&c.head, 3 * sizeof(int))) != cudaSuccess ||
            (e = cudaMemset(c.head, 0, 3 * sizeof(int))) != cudaSuccess ||
            (e = cudaHostAlloc(reinterpret_cast<void **>(&c.job_stage), sizeof(l2g::QueueJob) * (size_t)c.cap,
                               cudaHostAllocDefault)) != cudaSuccess ||
            (e = cudaHostAlloc(reinterpret_cast<void **>(&c.seg_stage), sizeof(l2g::Segment) * (size_t)s->nslots,
                               cudaHostAllocDefault)) != cudaSuccess ||
            (e = cudaHostAlloc(reinterpret_cast<void **>(&c.tail_stage), sizeof(int) * (size_t)c.ntail,
                               cudaHostAllocDefault)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&c.kst, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&c.fst, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&c.kev, cudaEventDisableTiming)) != cudaSuccess) {
            free_loop(s);
            return fail(std::string("pf_server_device_loop: allocation: ") + cudaGetErrorString(e));
        }
        c.tail = c.head + 1;
        c.closing = c.head + 2;
        std::memset(c.seg_stage, 0, sizeof(l2g::Segment) * (size_t)s->nslots);
        ++k;
    }
    s->loop = true;
    return 0;
}

int pf_server_configure(pf_server *s, int reserved_sms, int large_request_ctas) {
    if (!s || reserved_sms < 0 || large_request_ctas < 0) return fail("pf_server_configure: invalid argument");
    s->reserved_sms = std::min(reserved_sms, s->num_sms - 1);
    s->large_ctas = large_request_ctas > 0 ? large_request_ctas : (1 << 30);
    return 0;
}

int pf_server_latency_split(pf_server *s, int grid, int kind, double *out, int reset) {
    if (!s || grid < 0 || grid >= (int)s->grids.size() || (kind != 0 && kind != 1) || !out)
        return fail("pf_server_latency_split: invalid argument");
    std::vector<float> &w = s->wait_ms[2 * grid + kind], &d = s->run_ms[2 * grid + kind];
    out[0] = pct(w, 0.5);
    out[1] = pct(w, 0.99);
    out[2] = pct(d, 0.5);
    out[3] = pct(d, 0.99);
    out[4] = (double)d.size();
    if (reset) {
        w.clear();
        d.clear();
    }
    return 0;
}

int pf_server_state(const pf_server *s, int *pending, int *inflight, long long *bytes_in_use) {
    if (!s) return fail("pf_server_state: null argument");
    if (pending) *pending = (int)s->pending.size();
    if (inflight) {
        // on the device, or finished and not yet returned by pf_server_poll
        std::lock_guard<std::mutex> lk(s->mu);
        *inflight = (int)(s->inflight.size() + s->to_deliver.size() + s->delivered.size());
    }
    if (bytes_in_use) *bytes_in_use = (long long)s->in_use;
    return 0;
}

void pf_server_destroy(pf_server *s) {
    if (!s) return;
    for (Req *r : s->inflight) cudaEventSynchronize(s->slots[r->slot].ev);
    stop_workers(s);  // lets the workers finish the queued deliveries first
    destroy(s);
}

}  // extern "C"
