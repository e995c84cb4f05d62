// C ABI of the engine: plan lifetime, device upload, batch orchestration.
#include "../../include/lightsim2grid_b200.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <unistd.h>

#include "pf_capi_internal.hpp"
#include "pf_engine.cuh"
#include "pf_flows.cuh"
#include "pf_assembly.cuh"
#include "pf_plan.hpp"

using l2g::cplx;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *where) {
    g_err = std::string(where) + ": " + cudaGetErrorString(e);
    return -2;
}

// Host threads for the per-case preparation of large N-1 batches: a pool started on first use
// and kept for the life of the process (never joined: its threads sleep on a condition variable
// between calls).  One parallel region at a time; a caller that finds the pool busy (another
// host thread preparing a batch), or a process forked after the pool started (which has none of
// its threads), runs its region on its own thread.
class HostPool {
  public:
    static HostPool &get() {
        static HostPool *pool = new HostPool();
        return *pool;
    }
    int threads() const { return (int)workers_.size() + 1; }
    // fn(t, nt) for t = 0 .. nt-1, t = 0 on the calling thread
    void run(int nt, const std::function<void(int, int)> &fn) {
        nt = std::max(1, std::min(nt, threads()));
        if (getpid() != owner_) nt = 1;
        if (nt == 1) {
            fn(0, 1);
            return;
        }
        std::unique_lock<std::mutex> region(busy_, std::try_to_lock);
        if (!region.owns_lock()) {
            fn(0, 1);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(m_);
            job_ = &fn;
            njob_ = nt;
            pending_ = nt - 1;
            ++gen_;
        }
        cv_.notify_all();
        fn(0, nt);
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&] { return pending_ == 0; });
        job_ = nullptr;
    }

  private:
    HostPool() : owner_(getpid()) {
        const int hw = (int)std::thread::hardware_concurrency();
        const int nw = std::max(0, std::min(hw, 16) - 1);
        for (int i = 0; i < nw; ++i) {
            workers_.emplace_back([this, i] { loop(i + 1); });
            workers_.back().detach();
        }
    }
    void loop(int id) {
        long long seen = 0;
        std::unique_lock<std::mutex> lk(m_);
        for (;;) {
            cv_.wait(lk, [&] { return gen_ != seen; });
            seen = gen_;
            if (id >= njob_) continue;
            const std::function<void(int, int)> *f = job_;
            const int nt = njob_;
            lk.unlock();
            (*f)(id, nt);
            lk.lock();
            if (--pending_ == 0) done_.notify_one();
        }
    }
    pid_t owner_;
    std::vector<std::thread> workers_;
    std::mutex busy_, m_;
    std::condition_variable cv_, done_;
    const std::function<void(int, int)> *job_ = nullptr;
    int njob_ = 0, pending_ = 0;
    long long gen_ = 0;
};

// [lo, hi) of part t of nt equal parts of [0, n)
inline void part_range(int n, int t, int nt, int &lo, int &hi) {
    lo = (int)((long long)n * t / nt);
    hi = (int)((long long)n * (t + 1) / nt);
}

// Entry points that take device pointers launch on the current device: it must be the device the
// plan's structure and scratch live on (a plan is bound to the device current at its creation).
int check_plan_device(int plan_device, const char *who) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, who);
    if (dev != plan_device)
        return fail(-1, std::string(who) + ": the plan was built on device " + std::to_string(plan_device) +
                            " but device " + std::to_string(dev) + " is current");
    return 0;
}

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

}  // namespace

struct pf_plan {
    l2g::Plan P;
    pf_options opt{};
    int device = 0;
    int num_sms = 0;
    int precision = 0;
    int threads = 256;
    bool lu_in_smem = false;
    bool refine = false;
    int ctas_per_sm = 1;
    int grid = 1;
    size_t slab = 0, smem = 0;
    // mixed form: FP64 fallback inside launches on the plan's own scratch (slab and shared
    // memory sized for it), and whether the last launch ran it
    bool inline_fb = false, last_inline = false;
    size_t slab_fb = 0, smem_fb = 0;
    // device structure
    void *d_int = nullptr;
    void *d_dbl = nullptr;
    l2g::DevPlan dp{};
    // fast-decoupled plans: the B' and B'' systems
    l2g::DevPlan dsub[2]{};
    void *d_sub_int[2] = {nullptr, nullptr}, *d_sub_dbl[2] = {nullptr, nullptr};
    // batch-interleaved kernel: per-CTA slabs, hand-off lists and a row of ones (allocated on
    // first use)
    DevBuf tile_scratch, tile_aux;
    int tile_ones = 0;       // instances for which tile_aux holds the row of ones
    bool last_tile = false;  // the last launch ran the batch-interleaved kernel
    // device work buffers
    DevBuf scratch, counter, V0, Sbus, optr, opos, oval, jfirst, jcount, Vout, iters, errs, Jout, cycles, Vcase,
        casemap;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // result downloads that overlap the FP64 re-run
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // host state
    std::vector<double> lastJ;
    bool haveJ = false;
    double timers[6] = {0, 0, 0, 0, 0, 0};
    // islanding: undirected graph of off-diagonal entries with |y| > 1e-8 and its bridges
    std::vector<char> is_bridge_csr;  // per CSR position
    bool base_connected = false;
    bool graph_symmetric = true;
};

// A launch over several plans (pf_multi_create): segment table, scratch and job lists.
struct pf_multi {
    std::vector<pf_plan *> plans;
    int device = 0, precision = 0, threads = 0, grid = 0, num_sms = 0;
    bool lu_in_smem = false, refine = false;
    size_t smem = 0, slab = 0;
    DevBuf segs, scratch, counter;
    l2g::Segment seg0{};
    l2g::MultiArgs M{};
};

namespace {

// ------------------------------------------------------------------ islanding check
// Reference: ContingencyAnalysis::check_invertible (ContingencyAnalysis.cpp:14-45), a BFS from
// bus 0 that follows entries Y(r, c) with |y| > 1e-8 from column c to row r.
bool bfs_connected(const l2g::Plan &P, const std::vector<int> &opos, const std::vector<cplx> &oval) {
    const int n = P.n;
    std::vector<char> seen(n, 0);
    std::vector<int> queue;
    queue.reserve(n);
    // CSC traversal with overrides (positions are CSR; map through csr_of_csc)
    auto value_at_csc = [&](int p) {
        int d = P.csr_of_csc[p];
        for (size_t i = 0; i < opos.size(); ++i)
            if (opos[i] == d) return oval[i];
        return P.Rx[d];
    };
    seen[0] = 1;
    queue.push_back(0);
    for (size_t h = 0; h < queue.size(); ++h) {
        int c = queue[h];
        for (int p = P.Yp[c]; p < P.Yp[c + 1]; ++p) {
            int r = P.Yi[p];
            if (seen[r]) continue;
            if (std::abs(value_at_csc(p)) > 1e-8) {
                seen[r] = 1;
                queue.push_back(r);
            }
        }
    }
    return (int)queue.size() == n;
}

void compute_bridges(pf_plan *pl) {
    const l2g::Plan &P = pl->P;
    const int n = P.n;
    pl->is_bridge_csr.assign(P.nnzY, 0);
    // symmetric strong-entry graph?
    pl->graph_symmetric = true;
    std::vector<std::vector<std::pair<int, int>>> adj(n);  // (neighbour, CSR position of (r=u, c=v))
    for (int r = 0; r < n; ++r)
        for (int d = P.Rp[r]; d < P.Rp[r + 1]; ++d) {
            int c = P.Rj[d];
            if (c == r) continue;
            bool strong = std::abs(P.Rx[d]) > 1e-8;
            // transposed entry
            int dt = -1;
            for (int e = P.Rp[c]; e < P.Rp[c + 1]; ++e)
                if (P.Rj[e] == r) { dt = e; break; }
            bool strong_t = dt >= 0 && std::abs(P.Rx[dt]) > 1e-8;
            if (strong != strong_t) pl->graph_symmetric = false;
            if (strong && r < c) {
                adj[r].push_back({c, d});
                adj[c].push_back({r, d});
            }
        }
    std::vector<int> none, ops;
    std::vector<cplx> ovs;
    pl->base_connected = bfs_connected(P, ops, ovs);
    // Tarjan's bridge finding (iterative)
    std::vector<int> disc(n, -1), low(n, 0), parent_edge(n, -1), it(n, 0);
    int timer = 0;
    for (int s = 0; s < n; ++s) {
        if (disc[s] >= 0) continue;
        std::vector<int> st{s};
        disc[s] = low[s] = timer++;
        while (!st.empty()) {
            int u = st.back();
            if (it[u] < (int)adj[u].size()) {
                auto [v, d] = adj[u][it[u]++];
                if (d == parent_edge[u]) continue;
                if (disc[v] < 0) {
                    parent_edge[v] = d;
                    disc[v] = low[v] = timer++;
                    st.push_back(v);
                } else {
                    low[u] = std::min(low[u], disc[v]);
                }
            } else {
                st.pop_back();
                if (!st.empty()) {
                    int p = st.back();
                    low[p] = std::min(low[p], low[u]);
                    if (low[u] > disc[p]) pl->is_bridge_csr[parent_edge[u]] = 1;
                }
            }
        }
    }
}

int csr_find(const l2g::Plan &P, int r, int c) {
    if (r < 0 || r >= P.n || c < 0 || c >= P.n) return -1;
    const int *b = P.Rj.data() + P.Rp[r], *e = P.Rj.data() + P.Rp[r + 1];
    const int *f = std::lower_bound(b, e, c);
    if (f == e || *f != c) return -1;
    return (int)(f - P.Rj.data());
}

// overrides of one case; returns 0, or -1 if a coefficient is outside the pattern
int case_overrides(const l2g::Plan &P, int k0, int k1, const int *row, const int *col, const cplx *val,
                   std::vector<int> &opos, std::vector<cplx> &oval) {
    opos.clear();
    oval.clear();
    for (int k = k0; k < k1; ++k) {
        int d = csr_find(P, row[k], col[k]);
        if (d < 0) return -1;
        size_t i = 0;
        for (; i < opos.size(); ++i)
            if (opos[i] == d) break;
        if (i == opos.size()) {
            opos.push_back(d);
            oval.push_back(P.Rx[d]);
        }
        oval[i] -= val[k];
    }
    return 0;
}

bool case_connected(pf_plan *pl, const std::vector<int> &opos, const std::vector<cplx> &oval) {
    const l2g::Plan &P = pl->P;
    if (!pl->base_connected) return false;
    // edges of the strong graph turned off / on by this case
    int removed = 0, removed_pos = -1;
    bool added = false;
    for (size_t i = 0; i < opos.size(); ++i) {
        int d = opos[i];
        int r = P.Rrow[d], c = P.Rj[d];
        if (r == c) continue;
        bool before = std::abs(P.Rx[d]) > 1e-8, after = std::abs(oval[i]) > 1e-8;
        if (before && !after) {
            ++removed;
            if (r < c) removed_pos = d;
        }
        if (!before && after) added = true;
    }
    if (removed == 0 && !added) return true;
    if (pl->graph_symmetric && !added && removed == 2 && removed_pos >= 0) {
        // one undirected edge gone (both directions): connected unless it is a bridge
        int r = P.Rrow[removed_pos], c = P.Rj[removed_pos];
        bool other_gone = false;
        for (size_t i = 0; i < opos.size(); ++i)
            if (P.Rrow[opos[i]] == c && P.Rj[opos[i]] == r && !(std::abs(oval[i]) > 1e-8)) other_gone = true;
        if (other_gone) return !pl->is_bridge_csr[removed_pos];
    }
    return bfs_connected(P, opos, oval);
}

// ------------------------------------------------------------------ device upload
template <typename T>
size_t push(std::vector<unsigned char> &blob, const std::vector<T> &v) {
    size_t off = (blob.size() + 15) & ~(size_t)15;
    blob.resize(off + v.size() * sizeof(T));
    if (!v.empty()) std::memcpy(blob.data() + off, v.data(), v.size() * sizeof(T));
    return off;
}

std::vector<int> pack_pairs(const std::vector<int> &a, const std::vector<int> &b) {
    std::vector<int> out(2 * a.size());
    for (size_t i = 0; i < a.size(); ++i) {
        out[2 * i] = a[i];
        out[2 * i + 1] = b[i];
    }
    return out;
}

// Uploads the structure arrays of one plan (and, for a fast-decoupled system, its factor
// values) into two device blobs and points the fields of `d` into them.
int upload_plan(const l2g::Plan &P, l2g::DevPlan &d, void *&d_int, void *&d_dbl, const std::vector<double> *luval,
                int lu_offset = -1, bool compact_ok = true) {
    std::vector<unsigned char> bi, bd;
    size_t oRp = push(bi, P.Rp), oRj = push(bi, P.Rj), oRrow = push(bi, P.Rrow);
    size_t oyt = push(bi, P.ytarget), oyj = push(bi, P.yjpos);
    size_t ofill = push(bi, P.fillpos), ocpos = push(bi, P.cpos), ocj = push(bi, P.cjpos);
    size_t oxP = push(bi, P.xP), oxQ = push(bi, P.xQ), oxVa = push(bi, P.xVa), oxVm = push(bi, P.xVm);
    size_t ofo = push(bi, P.factor.ops), ofb = push(bi, P.factor.base), ofw = push(bi, P.factor.width);
    size_t obo = push(bi, P.backward.ops), obb = push(bi, P.backward.base), obw = push(bi, P.backward.width);
    size_t owo = push(bi, P.forward.ops), owb = push(bi, P.forward.base), oww = push(bi, P.forward.width);
    // packed operations for the shared-memory LU layout (always fit when the LU does)
    const bool compact = lu_offset >= 0 ? compact_ok : l2g::compact_fits(P);
    std::vector<unsigned> cf, cb, cw;
    if (compact) {
        l2g::compact_ops(P.factor, P.m, cf, lu_offset);
        l2g::compact_ops(P.backward, P.m, cb, lu_offset);
        l2g::compact_ops(P.forward, P.m, cw, lu_offset);
    }
    size_t ocf = push(bi, cf), ocb = push(bi, cb), ocw = push(bi, cw);
    // the programs regrouped for the batch-interleaved kernel (Newton plans)
    l2g::TileProgram tf, tb, tw;
    if (!P.dc && !P.fdpf) {
        l2g::build_tile_program(P.factor, l2g::kTileWarps, l2g::kTileChunk, tf);
        l2g::build_tile_program(P.backward, l2g::kTileWarps, l2g::kTileChunk, tb);
        l2g::build_tile_program(P.forward, l2g::kTileWarps, l2g::kTileChunk, tw);
        // padding becomes an update of the scratch LU row nnzLU (the kernel has no branch on it)
        for (l2g::TileProgram *t : {&tf, &tb, &tw})
            for (size_t o = 0; o < t->ops.size(); o += 4)
                if (((unsigned)t->ops[o + 3] >> 28) == 7u) {
                    t->ops[o] = t->ops[o + 1] = t->ops[o + 2] = P.nnzLU;
                    t->ops[o + 3] = P.nnzLU;
                }
    }
    size_t otfo = push(bi, tf.ops), otbo = push(bi, tb.ops), otwo = push(bi, tw.ops);
    size_t otfp = push(bi, tf.phase), otbp = push(bi, tb.phase), otwp = push(bi, tw.phase);
    size_t odpos = push(bi, P.dpos);
    size_t otail = push(bi, P.tail_map);
    std::vector<double> rx(2 * (size_t)P.nnzY);
    for (int i = 0; i < P.nnzY; ++i) {
        rx[2 * i] = P.Rx[i].real();
        rx[2 * i + 1] = P.Rx[i].imag();
    }
    // J(P(r), 0) of the distributed-slack Jacobian (BaseNRAlgo.tpp:542-552)
    std::vector<double> wJ(P.n, 0.0);
    if (P.distributed)
        for (int r = 0; r < P.n; ++r) {
            if (P.xP[r] < 0) continue;
            if (r == P.slack0) wJ[r] = P.weights[r];
            else if (std::fabs(P.weights[r]) > 1e-7) wJ[r] = P.weights[r];
        }
    size_t oRx = push(bd, rx), ow = push(bd, P.weights), ocv = push(bd, P.cval), owJ = push(bd, wJ);
    size_t olu = push(bd, luval ? *luval : std::vector<double>());
    if (d_int) cudaFree(d_int);
    if (d_dbl) cudaFree(d_dbl);
    d_int = d_dbl = nullptr;
    cudaError_t e = cudaMalloc(&d_int, std::max<size_t>(bi.size(), 16));
    if (e != cudaSuccess) return cuda_fail(e, "pf_plan_create: cudaMalloc");
    e = cudaMalloc(&d_dbl, std::max<size_t>(bd.size(), 16));
    if (e != cudaSuccess) return cuda_fail(e, "pf_plan_create: cudaMalloc");
    if (!bi.empty() && (e = cudaMemcpy(d_int, bi.data(), bi.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_fail(e, "pf_plan_create: upload");
    if (!bd.empty() && (e = cudaMemcpy(d_dbl, bd.data(), bd.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_fail(e, "pf_plan_create: upload");
    unsigned char *bI = static_cast<unsigned char *>(d_int), *bD = static_cast<unsigned char *>(d_dbl);
    auto I = [&](size_t o) { return reinterpret_cast<const int *>(bI + o); };
    auto I4 = [&](size_t o) { return reinterpret_cast<const int4 *>(bI + o); };
    auto D = [&](size_t o) { return reinterpret_cast<const double *>(bD + o); };
    d = l2g::DevPlan{};
    d.n = P.n;
    d.m = P.m;
    d.nnzY = P.nnzY;
    d.nnzLU = P.nnzLU;
    d.distributed = P.distributed ? 1 : 0;
    d.Rp = I(oRp);
    d.Rj = I(oRj);
    d.Rrow = I(oRrow);
    d.Rx = reinterpret_cast<const double2 *>(D(oRx));
    d.w = D(ow);
    d.ytarget = I4(oyt);
    d.yjpos = I4(oyj);
    d.fillpos = I(ofill);
    d.nfill = (int)P.fillpos.size();
    d.cpos = I(ocpos);
    d.cjpos = I(ocj);
    d.cval = D(ocv);
    d.nconst = (int)P.cpos.size();
    d.xP = I(oxP);
    d.xQ = I(oxQ);
    d.xVa = I(oxVa);
    d.xVm = I(oxVm);
    d.xSlack = P.xSlack;
    d.wJ = D(owJ);
    d.fac_ops = I4(ofo);
    d.fac_base = I(ofb);
    d.fac_width = I(ofw);
    d.bwd_width = I(obw);
    d.fwd_width = I(oww);
    auto U2 = [&](size_t o) { return reinterpret_cast<const uint2 *>(bI + o); };
    d.compact = compact ? 1 : 0;
    d.lu_offset = lu_offset >= 0 ? lu_offset : l2g::compact_lu_offset(P.m);
    d.fac_cops = compact ? U2(ocf) : nullptr;
    d.bwd_cops = compact ? U2(ocb) : nullptr;
    d.fwd_cops = compact ? U2(ocw) : nullptr;
    d.fac_nph = P.factor.nphases();
    d.bwd_ops = I4(obo);
    d.bwd_base = I(obb);
    d.bwd_nph = P.backward.nphases();
    d.fwd_ops = I4(owo);
    d.fwd_base = I(owb);
    d.fwd_nph = P.forward.nphases();
    d.dpos = I(odpos);
    d.dc = P.dc ? 1 : 0;
    d.slack0 = P.slack0;
    d.luval = luval ? D(olu) : nullptr;
    const bool tiled = !P.dc && !P.fdpf;
    d.tfac_ops = tiled ? I4(otfo) : nullptr;
    d.tbwd_ops = tiled ? I4(otbo) : nullptr;
    d.tfwd_ops = tiled ? I4(otwo) : nullptr;
    d.tfac_phase = tiled ? I(otfp) : nullptr;
    d.tbwd_phase = tiled ? I(otbp) : nullptr;
    d.tfwd_phase = tiled ? I(otwp) : nullptr;
    d.tail_ct = P.tail_k > 0 ? P.tail_ct : P.m;
    d.tail_k = P.tail_k;
    d.tail_map = P.tail_k > 0 ? I(otail) : nullptr;
    return 0;
}

// Narrow phases of the packed programs that run on a few warps with their operations staged in
// shared memory (DevPlan::nar_*): the factor's and the forward program's last phases and the
// backward program's first ones, each at most kNarrowThreads wide, as many as `budget` bytes
// of shared memory hold (factor first, then backward, then forward, each range grown from its
// narrow end).  A phase there costs shared-memory latency and a barrier of those warps instead
// of a block barrier that waits for the next operations' global loads.
constexpr int kNarrowThreads = 128;

void narrow_phases(const l2g::Plan &P, l2g::DevPlan &d, size_t budget) {
    for (int k = 0; k < 3; ++k) d.nar_a[k] = d.nar_b[k] = d.nar_first[k] = 0;
    for (int k = 0; k < 4; ++k) d.nar_off[k] = 0;
    d.nar_warps = 0;
    if (!d.compact) return;
    const size_t slack = 16;  // alignment of the staged area
    size_t left = budget > slack ? budget - slack : 0;
    const l2g::Plan::Program *pr[3] = {&P.factor, &P.backward, &P.forward};
    int widest = 0, off = 0;
    for (int k = 0; k < 3; ++k) {
        const l2g::Plan::Program &g = *pr[k];
        const int nph = g.nphases();
        int a = nph, b = nph;  // suffix [a, nph) for the factor and forward programs
        if (k == 1) a = b = 0;  // prefix [0, b) for the backward program
        for (;;) {
            const int p = k == 1 ? b : a - 1;
            if (p < 0 || p >= nph || g.width[p] > kNarrowThreads) break;
            const size_t bytes = (size_t)(g.base[p + 1] - g.base[p]) * 8;
            if (bytes > left) break;
            left -= bytes;
            widest = std::max(widest, g.width[p]);
            if (k == 1) ++b;
            else --a;
        }
        if (b - a < 2) a = b = 0;  // a single phase is not worth a range
        d.nar_a[k] = a;
        d.nar_b[k] = b;
        d.nar_first[k] = b > a ? g.base[a] : 0;
        d.nar_off[k] = off;
        off += b > a ? g.base[b] - g.base[a] : 0;
    }
    d.nar_off[3] = off;
    d.nar_warps = (widest + 31) / 32;
    if (off == 0) d.nar_warps = 0;
}

int upload(pf_plan *pl) {
    int rc = upload_plan(pl->P, pl->dp, pl->d_int, pl->d_dbl, nullptr);
    if (rc || !pl->P.fdpf) return rc;
    int off[2];
    bool fits = false;
    l2g::fdpf_lu_offsets(pl->P, off[0], off[1], fits);
    for (int k = 0; k < 2; ++k) {
        rc = upload_plan(pl->P.sub[k], pl->dsub[k], pl->d_sub_int[k], pl->d_sub_dbl[k], &pl->P.sublu[k], off[k],
                         fits);
        if (rc) return rc;
    }
    return 0;
}

// Mixed form: below which ||F||_inf a refined step reuses the previous iteration's LU
// (never above the refinement threshold; option <= 0: never).
double lu_reuse_below(const pf_plan *pl, double refine_below) {
    const double want = pl->opt.lu_reuse_threshold;
    return want <= 0 ? 0.0 : std::min(want, refine_below);
}

int configure(pf_plan *pl) {
    const l2g::Plan &P = pl->P;
    cudaError_t e = cudaGetDevice(&pl->device);
    if (e != cudaSuccess) return cuda_fail(e, "pf_plan_create: no CUDA device");
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, pl->device);
    if (e != cudaSuccess) return cuda_fail(e, "pf_plan_create: cudaGetDeviceProperties");
    pl->num_sms = prop.multiProcessorCount;
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, pl->device);
    pl->precision = pl->opt.precision ? 1 : 0;
    const int thr = pl->threads;
    if (P.fdpf) {
        // FP64; both factors in every CTA's shared memory when they fit
        pl->precision = 0;
        pl->refine = false;
        const size_t static_smem = 4096;  // Shared struct and the three staged plans
        const size_t sm_in = l2g::fdpf_smem_bytes(pl->dsub[0], pl->dsub[1], true);
        const size_t sm_out = l2g::fdpf_smem_bytes(pl->dsub[0], pl->dsub[1], false);
        const bool fits = pl->dsub[0].compact && pl->dsub[1].compact && sm_in + static_smem <= (size_t)optin;
        if (pl->opt.lu_placement == 1 && !fits) return fail(-1, "pf_plan_create: the factors do not fit in shared memory");
        if (sm_out + static_smem > (size_t)optin)
            return fail(-1, "pf_plan_create: the solve vectors do not fit in shared memory");
        pl->lu_in_smem = pl->opt.lu_placement == 2 ? false : fits;
        pl->smem = pl->lu_in_smem ? sm_in : sm_out;
        pl->slab = l2g::fdpf_slab_bytes(pl->dp);
        pl->slab_fb = pl->slab;
        pl->smem_fb = pl->smem;
        pl->inline_fb = false;
        const int want = pl->opt.max_ctas_per_sm;
        int occ = l2g::fdpf_occupancy(pl->lu_in_smem, thr, want > 0 ? want : 8, pl->smem);
        if (occ <= 0) return fail(-1, "pf_plan_create: the kernel cannot be launched with this configuration");
        if (want > 0) occ = std::min(occ, want);
        pl->ctas_per_sm = occ;
        pl->grid = pl->num_sms * occ;
        e = pl->scratch.ensure(pl->slab * (size_t)pl->grid);
        if (e != cudaSuccess) return cuda_fail(e, "pf_plan_create: scratch allocation");
        e = pl->counter.ensure(256);
        if (e != cudaSuccess) return cuda_fail(e, "pf_plan_create: counter allocation");
        return 0;
    }
    const int lub = pl->precision ? 4 : 8, xb = pl->precision ? 4 : 8;
    const size_t static_smem = 2048;  // Shared struct of the kernel, rounded up
    size_t sm_in = l2g::smem_bytes(pl->dp, lub, xb, true);
    size_t sm_out = l2g::smem_bytes(pl->dp, lub, xb, false);
    bool fits = pl->dp.compact && sm_in + static_smem <= (size_t)optin;
    if (pl->opt.lu_placement == 1 && !fits) return fail(-1, "pf_plan_create: LU does not fit in shared memory");
    if (sm_out + static_smem > (size_t)optin)
        return fail(-1, "pf_plan_create: the solve vector does not fit in shared memory");
    if (P.tail_k > 0 && pl->opt.lu_placement == 1)
        return fail(-1, "pf_plan_create: a plan with a dense tail keeps its LU in global memory");
    pl->lu_in_smem = pl->opt.lu_placement == 2 || P.tail_k > 0 ? false : fits;
    pl->smem = pl->lu_in_smem ? sm_in : sm_out;
    if (pl->lu_in_smem && thr <= 640) {  // the 768-thread kernel runs every phase block-wide
        narrow_phases(pl->P, pl->dp, (size_t)optin - static_smem - pl->smem);
        pl->smem = l2g::smem_bytes(pl->dp, lub, xb, true);
    }
    pl->slab = l2g::slab_bytes(pl->dp, lub, pl->lu_in_smem);
    pl->refine = pl->precision == 1 && pl->opt.refine != 2;
    int occ = l2g::nr_occupancy(pl->precision, pl->lu_in_smem, pl->refine, thr, pl->smem);
    if (occ <= 0) return fail(-1, "pf_plan_create: the kernel cannot be launched with this configuration");
    if (pl->opt.max_ctas_per_sm > 0) occ = std::min(occ, pl->opt.max_ctas_per_sm);
    pl->ctas_per_sm = occ;
    pl->grid = pl->num_sms * occ;
    // mixed form with refinement: the FP64 fallback runs inside launches on the plan's own
    // scratch, whose slabs then also hold an FP64 LU and whose shared memory an FP64 solve vector
    pl->slab_fb = pl->slab;
    pl->smem_fb = pl->smem;
    pl->inline_fb = false;
    if (pl->precision == 1 && pl->refine && pl->opt.fp64_fallback != 2) {
        const size_t sfb = std::max(pl->smem, l2g::smem_bytes(pl->dp, 8, 8, false));
        if (sfb + static_smem <= (size_t)optin &&
            l2g::nr_occupancy(pl->precision, pl->lu_in_smem, pl->refine, thr, sfb) >= pl->ctas_per_sm) {
            pl->inline_fb = true;
            pl->smem_fb = sfb;
            pl->slab_fb = std::max(pl->slab, l2g::slab_bytes(pl->dp, 8, false));
        }
    }
    e = pl->scratch.ensure(pl->slab_fb * (size_t)pl->grid);
    if (e != cudaSuccess) return cuda_fail(e, "pf_plan_create: scratch allocation");
    e = pl->counter.ensure(256);
    if (e != cudaSuccess) return cuda_fail(e, "pf_plan_create: counter allocation");
    return 0;
}

void release(pf_plan *pl) {
    for (DevBuf *b : {&pl->tile_scratch, &pl->tile_aux, &pl->scratch, &pl->counter, &pl->V0, &pl->Sbus, &pl->optr, &pl->opos, &pl->oval,
                      &pl->jfirst, &pl->jcount, &pl->Vout, &pl->iters, &pl->errs, &pl->Jout, &pl->cycles,
                      &pl->Vcase, &pl->casemap})
        b->release();
    if (pl->d_int) cudaFree(pl->d_int);
    if (pl->d_dbl) cudaFree(pl->d_dbl);
    pl->d_int = pl->d_dbl = nullptr;
    for (int k = 0; k < 2; ++k) {
        if (pl->d_sub_int[k]) cudaFree(pl->d_sub_int[k]);
        if (pl->d_sub_dbl[k]) cudaFree(pl->d_sub_dbl[k]);
        pl->d_sub_int[k] = pl->d_sub_dbl[k] = nullptr;
    }
    if (pl->ev0) cudaEventDestroy(pl->ev0);
    if (pl->ev1) cudaEventDestroy(pl->ev1);
    if (pl->stream) cudaStreamDestroy(pl->stream);
    if (pl->copy_stream) cudaStreamDestroy(pl->copy_stream);
    pl->copy_stream = nullptr;
    pl->ev0 = pl->ev1 = nullptr;
    pl->stream = nullptr;
}

// Launches the kernel for a batch whose device buffers are set up in `a` (no sync), with
// the per-CTA slabs in `scratch` (`scratch_bytes` long) and the job counter at `counter`.
// The number of CTAs is bounded by the slabs that fit in the scratch.
// Whether a launch runs the batch-interleaved kernel: Newton plans, independent instances (no
// chain), no per-launch diagnostics (J output, phase cycles or trace, LU reuse), and option
// batch_layout 2, or auto (0) for plans whose LU stays in global memory and has at least
// kAutoTileLU entries, with several jobs per SM.  Measured on all N-1 outages: 6,515 buses mixed
// 74.4 against 85.7 ms (one 768-thread CTA per instance), FP64 70 against 107 ms; 2,848 buses FP64
// (48,682 LU entries) 17.6 against 17.5 ms, so it stays on one CTA per instance.  Where the LU
// sits in shared memory (up to 2,848 buses mixed, 1,354 buses FP64) one CTA per instance is
// faster (2,848 mixed: 9.4 against 20.4 ms).
constexpr int kAutoTileLU = 60000;

bool use_tile(const pf_plan *pl, const l2g::BatchArgs &a) {
    if (pl->P.dc || pl->P.fdpf || a.chain || a.Jout || a.trace || a.reuse_below > 0) return false;
    if (pl->P.tail_k > 0) return false;  // the dense tail runs in the one-CTA kernel
    if (pl->opt.batch_layout == 2) return true;
    return pl->opt.batch_layout == 0 && !pl->lu_in_smem && pl->P.nnzLU >= kAutoTileLU && a.njobs >= 4 * pl->num_sms;
}

int launch_into(pf_plan *pl, l2g::BatchArgs a, int precision, cudaStream_t st, unsigned char *scratch,
                size_t scratch_bytes, int *counter, bool allow_tile, bool allow_inline);

// The batch-interleaved kernel, then the one-CTA kernel over what it handed off: its stragglers
// (continued from their state) and, in the mixed form, its FP32 failures (re-solved in FP64 from
// their start voltages).  The lists and their counts stay in device memory: no host
// synchronisation.  Counter words: [0] jobs, [2] stragglers, [3] FP32 failures, [8..9] and [12..13]
// the two follow-up launches.
int launch_tile(pf_plan *pl, l2g::BatchArgs a, int precision, cudaStream_t st, int *counter) {
    const int lub = precision ? 4 : 8;
    const size_t slab = l2g::tile_slab_bytes(pl->dp, lub);
    const int grid = std::max(1, std::min(pl->num_sms, a.njobs));
    cudaError_t e = pl->tile_scratch.ensure(slab * (size_t)grid);
    if (e != cudaSuccess) return cuda_fail(e, "launch: batch-interleaved scratch allocation");
    const int ni = std::max(a.n_inst, 1);
    e = pl->tile_aux.ensure((size_t)3 * ni * sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "launch: batch-interleaved hand-off lists");
    int *hand = static_cast<int *>(pl->tile_aux.p), *fbl = hand + ni, *ones = hand + 2 * (size_t)ni;
    if (pl->tile_ones < ni) {
        std::vector<int> one((size_t)ni, 1);
        e = cudaMemcpyAsync(ones, one.data(), (size_t)ni * sizeof(int), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "launch: batch-interleaved job counts");
        pl->tile_ones = ni;
    }
    const l2g::BatchArgs orig = a;
    a.scratch = static_cast<unsigned char *>(pl->tile_scratch.p);
    a.slab_bytes = (long long)slab;
    a.job_counter = counter;
    // spread the jobs over all CTAs: lanes per CTA
    a.tile_lanes = std::max(1, std::min(32, (a.njobs + grid - 1) / grid));
    // hand-off point: with at most one job per lane (no refill) as soon as the jobs are exhausted,
    // i.e. after the first instance of the CTA finishes (2,848 buses, 21 lanes: FP64 20.8 -> 18.4
    // ms); with refills once half the lanes are idle (6,515 buses, 32 lanes: 77.1 ms mixed against
    // 78.6 when handing off at 24 lanes and 89.9 at 4)
    const int ho = pl->opt.handoff_lanes;
    a.hand_list = ho < 0 ? nullptr : hand;
    a.hand_count = counter + 2;
    const bool refills = (long long)a.njobs > (long long)grid * a.tile_lanes;
    a.hand_lanes = ho > 0 ? ho : (refills ? std::max(1, a.tile_lanes / 2) : a.tile_lanes);
    const bool fallback = precision == 1 && pl->precision == 1 && pl->opt.fp64_fallback != 2 && a.refine;
    a.fb_list = fallback ? fbl : nullptr;
    a.fb_count = counter + 3;
    e = cudaMemsetAsync(counter, 0, 16 * sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "launch: counter reset");
    e = l2g::launch_nr_tile(pl->dp, a, precision, grid, st);
    if (e != cudaSuccess) return cuda_fail(e, "launch: batch-interleaved kernel");
    // the stragglers, from their output rows and iteration counts (the mixed form's in-launch FP64
    // fallback covers their failures)
    l2g::BatchArgs c = orig;
    c.phase_cycles = nullptr;  // the per-section cycles are the interleaved kernel's
    c.job_first = hand;
    c.job_count = ones;
    c.njobs = a.n_inst;
    c.njobs_dev = counter + 2;
    c.it_start = a.iters;
    c.v0_from_out = 1;
    int rc = launch_into(pl, c, precision, st, static_cast<unsigned char *>(pl->scratch.p),
                         pl->slab_fb * (size_t)pl->grid, counter + 8, false, true);
    if (rc) return rc;
    if (fallback) {
        l2g::BatchArgs f = orig;
        f.phase_cycles = nullptr;
        f.job_first = fbl;
        f.job_count = ones;
        f.njobs = a.n_inst;
        f.njobs_dev = counter + 3;
        rc = launch_into(pl, f, 0, st, static_cast<unsigned char *>(pl->scratch.p), pl->slab_fb * (size_t)pl->grid,
                         counter + 12, false, false);
        if (rc) return rc;
    }
    pl->last_inline = fallback;
    pl->last_tile = true;
    return 0;
}

int launch_into(pf_plan *pl, l2g::BatchArgs a, int precision, cudaStream_t st, unsigned char *scratch,
                size_t scratch_bytes, int *counter, bool allow_tile = false, bool allow_inline = false) {
    pl->last_tile = false;
    a.scratch = scratch;
    a.slab_bytes = (long long)pl->slab;
    a.job_counter = counter;
    a.lu_in_smem = pl->lu_in_smem ? 1 : 0;
    a.refine = (precision == 1 && pl->refine) ? 1 : 0;
    a.refine_below = pl->opt.refine_threshold > 0 ? pl->opt.refine_threshold : 1e-3;
    a.reuse_below = lu_reuse_below(pl, a.refine_below);
    pl->last_inline = false;
    if (a.njobs <= 0) return 0;
    if (allow_tile && use_tile(pl, a)) return launch_tile(pl, a, precision, st, counter);
    if ((allow_tile || allow_inline) && pl->inline_fb && precision == pl->precision && a.refine && !pl->P.dc &&
        !pl->P.fdpf) {
        // the plan's own scratch: FP64 fallback inside the launch
        a.fp64_inline = 1;
        a.slab_bytes = (long long)pl->slab_fb;
        // the job counter and, after it, the count of instances re-solved in FP64
        cudaError_t e = cudaMemsetAsync(counter, 0, 2 * sizeof(int), st);
        if (e != cudaSuccess) return cuda_fail(e, "launch: counter reset");
        int grid = std::min(pl->grid, a.njobs);
        grid = std::min<long long>(grid, (long long)(scratch_bytes / pl->slab_fb));
        if (grid <= 0) return fail(-1, "launch: the scratch memory holds no CTA slab");
        e = l2g::launch_nr_batch(pl->dp, a, precision, pl->threads, grid, pl->smem_fb, st);
        if (e != cudaSuccess) return cuda_fail(e, "launch: kernel");
        pl->last_inline = true;
        return 0;
    }
    if (scratch_bytes < pl->slab) return fail(-1, "launch: the scratch memory holds no CTA slab");
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "launch: counter reset");
    int grid = std::min(pl->grid, a.njobs);
    grid = std::min<long long>(grid, (long long)(scratch_bytes / pl->slab));
    if (pl->P.fdpf) {
        e = l2g::launch_fdpf_batch(pl->dp, pl->dsub[0], pl->dsub[1], a, pl->threads, pl->ctas_per_sm, grid,
                                   pl->smem, st);
        if (e != cudaSuccess) return cuda_fail(e, "launch: kernel");
        return 0;
    }
    // the FP64 re-run of a mixed plan uses the FP64 kernel with this plan's layout:
    // LU bytes differ, so recompute shared memory and slab use for that precision
    size_t smem = pl->smem;
    int lub = precision ? 4 : 8;
    if (precision != pl->precision) {
        bool in = pl->lu_in_smem;
        size_t need = l2g::smem_bytes(pl->dp, lub, lub, in);
        size_t slab = l2g::slab_bytes(pl->dp, lub, in);
        int optin = 0;
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, pl->device);
        if (in && (need + 2048 > (size_t)optin || !pl->dp.compact)) {
            in = false;
            need = l2g::smem_bytes(pl->dp, lub, lub, false);
            slab = l2g::slab_bytes(pl->dp, lub, false);
        }
        if (slab > scratch_bytes) return fail(-1, "launch: the scratch memory holds no FP64 CTA slab");
        grid = std::max(1, std::min(grid, (int)(scratch_bytes / slab)));
        a.slab_bytes = (long long)slab;
        a.lu_in_smem = in ? 1 : 0;
        smem = need;
        int occ = l2g::nr_occupancy(precision, in, false, pl->threads, smem);
        if (occ <= 0) return fail(-1, "launch: FP64 re-run configuration cannot launch");
        grid = std::min(grid, pl->num_sms * occ);
    }
    e = l2g::launch_nr_batch(pl->dp, a, precision, pl->threads, grid, smem, st);
    if (e != cudaSuccess) return cuda_fail(e, "launch: kernel");
    return 0;
}

int launch(pf_plan *pl, l2g::BatchArgs a, int precision, cudaStream_t st) {
    return launch_into(pl, a, precision, st, static_cast<unsigned char *>(pl->scratch.p),
                       pl->slab_fb * (size_t)pl->grid, static_cast<int *>(pl->counter.p), true, true);
}

template <typename T>
cudaError_t h2d(DevBuf &b, const T *src, size_t count, cudaStream_t st) {
    cudaError_t e = b.ensure(count * sizeof(T));
    if (e != cudaSuccess || count == 0) return e;
    return cudaMemcpyAsync(b.p, src, count * sizeof(T), cudaMemcpyHostToDevice, st);
}

// runs instances [0, n_inst) described by host arrays; results into host arrays.
// V0: shared (v0_stride 0) or per instance; Sbus likewise.
// Where a batch writes its voltage rows when not into the plan's device buffer: `vout` (device
// address, e.g. of mapped host memory), row `rows[i]` for instance i, zero rows for instances
// that did not converge; `during` runs on the host while the kernel runs.
struct RowsOut {
    double2 *vout = nullptr;
    const int *rows = nullptr;
    const std::function<void()> *during = nullptr;
};

int run_batch(pf_plan *pl, int n_inst, const cplx *V0, long long v0_stride, const cplx *Sbus, long long sbus_stride,
              const std::vector<int> &optr, const std::vector<int> &opos, const std::vector<cplx> &oval,
              const std::vector<int> &jfirst, const std::vector<int> &jcount, int chain, int max_iter, double tol,
              cplx *Vout, int *iters, int *errs, bool want_J,
              const std::function<int(const std::vector<char> &)> *settled = nullptr,
              const RowsOut *rows_out = nullptr) {
    const int n = pl->P.n;
    cudaStream_t st = pl->stream;
    double t0 = now();
    cudaError_t e;
    size_t nv0 = v0_stride ? (size_t)n_inst * n : (size_t)n;
    size_t nsb = sbus_stride ? (size_t)n_inst * n : (size_t)n;
    if ((e = h2d(pl->V0, V0, nv0, st)) != cudaSuccess) return cuda_fail(e, "batch: V0 upload");
    if ((e = h2d(pl->Sbus, Sbus, nsb, st)) != cudaSuccess) return cuda_fail(e, "batch: Sbus upload");
    bool have_ovr = !optr.empty();
    if (have_ovr) {
        if ((e = h2d(pl->optr, optr.data(), optr.size(), st)) != cudaSuccess) return cuda_fail(e, "batch: upload");
        if ((e = h2d(pl->opos, opos.data(), opos.size(), st)) != cudaSuccess) return cuda_fail(e, "batch: upload");
        if ((e = h2d(pl->oval, oval.data(), oval.size(), st)) != cudaSuccess) return cuda_fail(e, "batch: upload");
    }
    if ((e = h2d(pl->jfirst, jfirst.data(), jfirst.size(), st)) != cudaSuccess) return cuda_fail(e, "batch: upload");
    if ((e = h2d(pl->jcount, jcount.data(), jcount.size(), st)) != cudaSuccess) return cuda_fail(e, "batch: upload");
    if (!rows_out && (e = pl->Vout.ensure((size_t)n_inst * n * sizeof(cplx))) != cudaSuccess)
        return cuda_fail(e, "batch: alloc");
    if ((e = pl->iters.ensure((size_t)n_inst * sizeof(int))) != cudaSuccess) return cuda_fail(e, "batch: alloc");
    if ((e = pl->errs.ensure((size_t)n_inst * sizeof(int))) != cudaSuccess) return cuda_fail(e, "batch: alloc");
    if (want_J && (e = pl->Jout.ensure(pl->P.Ji.size() * sizeof(double))) != cudaSuccess)
        return cuda_fail(e, "batch: alloc");
    double t1 = now();
    l2g::BatchArgs a{};
    a.n_inst = n_inst;
    a.V0 = static_cast<const double2 *>(pl->V0.p);
    a.v0_stride = v0_stride;
    a.Sbus = static_cast<const double2 *>(pl->Sbus.p);
    a.sbus_stride = sbus_stride;
    a.ovr_ptr = have_ovr ? static_cast<const int *>(pl->optr.p) : nullptr;
    a.ovr_pos = have_ovr ? static_cast<const int *>(pl->opos.p) : nullptr;
    a.ovr_val = have_ovr ? static_cast<const double2 *>(pl->oval.p) : nullptr;
    a.max_iter = max_iter;
    a.tol = tol;
    a.job_first = static_cast<const int *>(pl->jfirst.p);
    a.job_count = static_cast<const int *>(pl->jcount.p);
    a.njobs = (int)jfirst.size();
    a.chain = chain;
    a.Vout = rows_out ? rows_out->vout : static_cast<double2 *>(pl->Vout.p);
    if (rows_out) {
        a.vout_row = rows_out->rows;
        a.zero_failed = 1;
    }
    a.iters = static_cast<int *>(pl->iters.p);
    a.errs = static_cast<int *>(pl->errs.p);
    a.Jout = want_J ? static_cast<double *>(pl->Jout.p) : nullptr;
    a.j_inst = 0;
    cudaEventRecord(pl->ev0, st);
    int rc = launch(pl, a, pl->precision, st);
    if (rc) return rc;
    cudaEventRecord(pl->ev1, st);
    // host work that overlaps the kernel (before any copy that would wait for it)
    if (rows_out && rows_out->during) (*rows_out->during)();
    if ((e = cudaMemcpyAsync(iters, pl->iters.p, (size_t)n_inst * sizeof(int), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
        return cuda_fail(e, "batch: download");
    if ((e = cudaMemcpyAsync(errs, pl->errs.p, (size_t)n_inst * sizeof(int), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
        return cuda_fail(e, "batch: download");
    int words[16] = {0};  // the launch's counters: re-solves in FP64 done on the device
    if (pl->last_inline &&
        (e = cudaMemcpyAsync(words, pl->counter.p, sizeof(words), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "batch: download");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "batch: kernel execution");
    float kms = 0.f;
    cudaEventElapsedTime(&kms, pl->ev0, pl->ev1);
    double kernel_s = kms * 1e-3;
    // mixed form: re-run in FP64 the jobs that contain a failure.  `settled` (if given) is called
    // once the re-run is queued, with the instances it recomputes: every other instance's row is
    // final, so the caller can copy those rows out while the re-run runs.
    int rerun = pl->last_tile ? words[3] + words[9] : words[1];
    std::vector<char> again;
    if (settled) again.assign((size_t)n_inst, 0);
    if (pl->precision == 1 && pl->opt.fp64_fallback != 2 && !pl->last_inline) {
        std::vector<int> rf, rc2;
        for (size_t j = 0; j < jfirst.size(); ++j) {
            bool bad = false;
            for (int s = 0; s < jcount[j]; ++s)
                if (errs[jfirst[j] + s] != 0) bad = true;
            if (bad) {
                rf.push_back(jfirst[j]);
                rc2.push_back(jcount[j]);
                rerun += jcount[j];
                if (settled)
                    for (int s = 0; s < jcount[j]; ++s) again[(size_t)jfirst[j] + s] = 1;
            }
        }
        if (!rf.empty()) {
            if ((e = h2d(pl->jfirst, rf.data(), rf.size(), st)) != cudaSuccess) return cuda_fail(e, "rerun: upload");
            if ((e = h2d(pl->jcount, rc2.data(), rc2.size(), st)) != cudaSuccess) return cuda_fail(e, "rerun: upload");
            a.job_first = static_cast<const int *>(pl->jfirst.p);
            a.job_count = static_cast<const int *>(pl->jcount.p);
            a.njobs = (int)rf.size();
            cudaEventRecord(pl->ev0, st);
            rc = launch(pl, a, 0, st);
            if (rc) return rc;
            cudaEventRecord(pl->ev1, st);
            if (settled && (rc = (*settled)(again)) != 0) return rc;
            settled = nullptr;
            if ((e = cudaMemcpyAsync(iters, pl->iters.p, (size_t)n_inst * sizeof(int), cudaMemcpyDeviceToHost,
                                     st)) != cudaSuccess)
                return cuda_fail(e, "rerun: download");
            if ((e = cudaMemcpyAsync(errs, pl->errs.p, (size_t)n_inst * sizeof(int), cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess)
                return cuda_fail(e, "rerun: download");
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "rerun: kernel execution");
            cudaEventElapsedTime(&kms, pl->ev0, pl->ev1);
            kernel_s += kms * 1e-3;
        }
    }
    if (settled && (rc = (*settled)(again)) != 0) return rc;
    double t2 = now();
    if (Vout &&
        (e = cudaMemcpyAsync(Vout, pl->Vout.p, (size_t)n_inst * n * sizeof(cplx), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess)
        return cuda_fail(e, "batch: download");
    if (want_J) {
        pl->lastJ.resize(pl->P.Ji.size());
        if ((e = cudaMemcpyAsync(pl->lastJ.data(), pl->Jout.p, pl->lastJ.size() * sizeof(double),
                                 cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return cuda_fail(e, "batch: download");
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "batch: download");
    double t3 = now();
    pl->timers[2] = t1 - t0;
    pl->timers[3] = kernel_s;
    pl->timers[4] = t3 - t2;
    pl->timers[5] = rerun;
    return 0;
}

}  // namespace

// ------------------------------------------------------------------ internal (pf_capi_internal.hpp)
namespace l2g {

BatchArgs device_args(const pf_device_batch *b) {
    BatchArgs a{};
    a.n_inst = b->n_inst;
    a.V0 = static_cast<const double2 *>(b->V0);
    a.v0_stride = b->v0_stride;
    a.Sbus = static_cast<const double2 *>(b->Sbus);
    a.sbus_stride = b->sbus_stride;
    a.ovr_ptr = b->ovr_ptr;
    a.ovr_pos = b->ovr_pos;
    a.ovr_val = static_cast<const double2 *>(b->ovr_val);
    a.max_iter = b->max_iter;
    a.tol = b->tol;
    a.job_first = b->job_first;
    a.job_count = b->job_count;
    a.njobs = b->njobs;
    a.chain = b->chain;
    a.Vout = static_cast<double2 *>(b->Vout);
    a.iters = b->iters;
    a.errs = b->errs;
    a.Jout = nullptr;
    a.j_inst = -1;
    return a;
}

int batch_device_with_scratch(pf_plan *pl, const pf_device_batch *b, void *stream, void *scratch,
                              size_t scratch_bytes, bool fp64_fallback) {
    if (!pl || !b || !scratch) return fail(-1, "batch with scratch: null argument");
    if (int rc = check_plan_device(pl->device, "batch with scratch")) return rc;
    if (reinterpret_cast<uintptr_t>(scratch) % 256 != 0)
        return fail(-1, "batch with scratch: scratch not 256-byte aligned");
    const size_t head = 256;  // job counter
    if (scratch_bytes < head + pl->slab) return fail(-1, "batch with scratch: scratch holds no CTA slab");
    unsigned char *base = static_cast<unsigned char *>(scratch);
    l2g::BatchArgs a = l2g::device_args(b);
    if (fp64_fallback && pl->inline_fb && scratch_bytes < head + pl->slab_fb)
        return fail(-1, "batch with scratch: scratch holds no CTA slab with room for the FP64 fallback");
    return launch_into(pl, a, pl->precision, static_cast<cudaStream_t>(stream), base + head, scratch_bytes - head,
                       reinterpret_cast<int *>(base), false, fp64_fallback);
}

size_t plan_slab_bytes(const pf_plan *pl) { return pl ? pl->slab : 0; }

size_t plan_fallback_slab_bytes(const pf_plan *pl) { return pl ? (pl->inline_fb ? pl->slab_fb : pl->slab) : 0; }

int loop_shape(pf_plan *const *plans, int n, LoopShape *sh) {
    if (!plans || n <= 0 || !sh) return fail(-1, "request loop: invalid argument");
    LoopShape r;
    r.inline_fb = true;
    for (int i = 0; i < n; ++i) {
        const pf_plan *pl = plans[i];
        if (!pl) return fail(-1, "request loop: null plan");
        if (pl->P.dc || pl->P.fdpf) return fail(-1, "request loop: Newton plans only");
        if (i == 0) {
            r.device = pl->device;
            r.precision = pl->precision;
            r.refine = pl->refine;
            r.lu_in_smem = pl->lu_in_smem;
            r.num_sms = pl->num_sms;
        } else if (pl->device != r.device || pl->precision != r.precision || pl->refine != r.refine ||
                   pl->lu_in_smem != r.lu_in_smem) {
            return fail(-1, "request loop: plans differ in device, precision, refinement or LU placement");
        }
        r.inline_fb = r.inline_fb && pl->inline_fb;
        r.threads = std::max(r.threads, pl->threads);
    }
    for (int i = 0; i < n; ++i) {
        const pf_plan *pl = plans[i];
        r.smem = std::max(r.smem, r.inline_fb ? pl->smem_fb : pl->smem);
        r.slab = std::max(r.slab, r.inline_fb ? pl->slab_fb : pl->slab);
    }
    r.ctas_per_sm = l2g::nr_occupancy(r.precision, r.lu_in_smem, r.refine, r.threads, r.smem);
    if (r.ctas_per_sm <= 0) return fail(-1, "request loop: the plans' largest layout cannot be launched");
    *sh = r;
    return 0;
}

int loop_segment(pf_plan *pl, const pf_device_batch *b, const LoopShape &sh, unsigned char *scratch, Segment *seg) {
    if (!pl || !b || !seg || !scratch) return fail(-1, "request loop: invalid argument");
    Segment &sg = *seg;
    sg.P = pl->dp;
    sg.A = device_args(b);
    sg.A.scratch = scratch;
    sg.A.slab_bytes = (long long)sh.slab;
    sg.A.job_counter = nullptr;  // jobs come from the queue
    sg.A.lu_in_smem = sh.lu_in_smem ? 1 : 0;
    sg.A.refine = sh.refine ? 1 : 0;
    sg.A.refine_below = pl->opt.refine_threshold > 0 ? pl->opt.refine_threshold : 1e-3;
    sg.A.reuse_below = lu_reuse_below(pl, sg.A.refine_below);
    sg.A.fp64_inline = (sh.inline_fb && sh.refine && sh.precision == 1) ? 1 : 0;
    return 0;
}

int loop_launch(const LoopShape &sh, const Segment &seg0, const DevQueue &q, int grid, void *stream) {
    MultiArgs M{};
    M.q = q;
    l2g::BatchArgs a0 = seg0.A;
    a0.phase_cycles = nullptr;
    a0.trace = nullptr;
    cudaError_t e = l2g::launch_nr_batch(seg0.P, a0, sh.precision, sh.threads, grid, sh.smem,
                                         static_cast<cudaStream_t>(stream), M);
    if (e != cudaSuccess) return cuda_fail(e, "request loop: kernel");
    return 0;
}

int plan_device(const pf_plan *pl) { return pl ? pl->device : -1; }

void set_last_error(const std::string &msg) { g_err = msg; }

}  // namespace l2g

// Shared tail of plan creation: islanding data, stream, device upload, launch configuration.
int finish_plan(pf_plan *pl, pf_plan **out) {
    compute_bridges(pl);
    cudaError_t e = cudaStreamCreateWithFlags(&pl->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&pl->copy_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        if (pl->stream) cudaStreamDestroy(pl->stream);
        delete pl;
        return cuda_fail(e, "pf_plan_create: stream");
    }
    cudaEventCreate(&pl->ev0);
    cudaEventCreate(&pl->ev1);
    int rc = upload(pl);
    if (!rc) rc = configure(pl);
    if (rc) {
        std::string keep = g_err;
        release(pl);
        delete pl;
        g_err = keep;
        return rc;
    }
    *out = pl;
    return 0;
}

extern "C" {

// Level preference of minimum degree for options `o`: none for orderings 1 and 3, else
// o.level_slack when positive, 2 by default (a negative value also turns it off).
static int level_slack_of(const pf_options &o) {
    if (o.ordering == 1 || o.ordering == 3 || o.level_slack < 0) return 0;
    return o.level_slack > 0 ? std::min(o.level_slack, 64) : 2;
}

const char *pf_last_error(void) { return g_err.c_str(); }

int pf_plan_create(int n, const int *colptr, const int *rowind, const double *ybus_ri, const double *V0_ri,
                   const double *Sbus_ri, const int *slack_ids, int nslack, const double *slack_weights,
                   const int *pv, int npv, const int *pq, int npq, int distributed, const pf_options *opts,
                   pf_plan **out) {
    if (!out || !colptr || !rowind || !ybus_ri || !V0_ri || !Sbus_ri || !slack_ids || !slack_weights ||
        (npv && !pv) || (npq && !pq))
        return fail(-1, "pf_plan_create: null argument");
    *out = nullptr;
    pf_plan *pl = new pf_plan();
    if (opts) pl->opt = *opts;
    l2g::PlanOptions po;
    if (pl->opt.pivot_threshold > 0) po.pivot_threshold = pl->opt.pivot_threshold;
    po.order_trials = pl->opt.ordering == 1 ? 0 : (pl->opt.ordering == 2 ? 1 : 8);
    po.level_slack = level_slack_of(pl->opt);
    po.elem_bytes = pl->opt.precision ? 4 : 8;
    po.spread_clusters = pl->opt.placement != 2;
    {
        const int m_est = npv + (distributed && nslack > 1 ? nslack - 1 : 0) + 2 * npq + (distributed ? 1 : 0);
        int thr = pl->opt.threads;
        // the largest plans run 640 (mixed form) or 768 threads (FP64 form)
        if (thr <= 0)
            thr = m_est > 4000 ? (pl->opt.precision ? 640 : 768) : (m_est > 2000 ? 512 : (m_est > 300 ? 256 : 128));
        thr = std::max(32, std::min(768, (thr / 32) * 32));
        po.threads = thr;
        pl->threads = thr;
    }
    po.fuse_forward = pl->opt.fuse_forward != 2;
    std::string msg;
    int rc;
    try {
        rc = l2g::build_plan(pl->P, n, colptr, rowind, reinterpret_cast<const cplx *>(ybus_ri),
                             reinterpret_cast<const cplx *>(V0_ri), reinterpret_cast<const cplx *>(Sbus_ri),
                             slack_ids, nslack, slack_weights, pv, npv, pq, npq, distributed != 0, po, msg);
    } catch (const std::exception &ex) {
        rc = -1;
        msg = std::string("pf_plan_create: ") + ex.what();
    }
    if (rc != 0) {
        delete pl;
        return fail(rc, msg);
    }
    return finish_plan(pl, out);
}

int pf_dc_plan_create(int n, const int *colptr, const int *rowind, const double *ybus_ri, const int *slack_ids,
                      int nslack, const int *pv, int npv, const int *pq, int npq, const pf_options *opts,
                      pf_plan **out) {
    if (!out || !colptr || !rowind || !ybus_ri || !slack_ids || (npv && !pv) || (npq && !pq))
        return fail(-1, "pf_dc_plan_create: null argument");
    *out = nullptr;
    pf_plan *pl = new pf_plan();
    if (opts) pl->opt = *opts;
    pl->opt.precision = 0;  // the reference's DC solve is FP64
    l2g::PlanOptions po;
    if (pl->opt.pivot_threshold > 0) po.pivot_threshold = pl->opt.pivot_threshold;
    po.order_trials = pl->opt.ordering == 1 ? 0 : (pl->opt.ordering == 2 ? 1 : 8);
    po.level_slack = level_slack_of(pl->opt);
    po.elem_bytes = pl->opt.precision ? 4 : 8;
    po.spread_clusters = pl->opt.placement != 2;
    int thr = pl->opt.threads;
    if (thr <= 0) thr = n > 2000 ? 512 : (n > 300 ? 256 : 128);
    thr = std::max(32, std::min(512, (thr / 32) * 32));
    po.threads = pl->threads = thr;
    po.fuse_forward = true;
    std::string msg;
    int rc;
    try {
        rc = l2g::build_dc_plan(pl->P, n, colptr, rowind, reinterpret_cast<const cplx *>(ybus_ri), slack_ids, nslack,
                                pv, npv, pq, npq, po, msg);
    } catch (const std::exception &ex) {
        rc = -1;
        msg = std::string("pf_dc_plan_create: ") + ex.what();
    }
    if (rc != 0) {
        delete pl;
        return fail(rc, msg);
    }
    return finish_plan(pl, out);
}

int pf_fdpf_plan_create(int n, const int *colptr, const int *rowind, const double *ybus_ri, const int *bp_colptr,
                        const int *bp_rowind, const double *bp_x, const int *bpp_colptr, const int *bpp_rowind,
                        const double *bpp_x, const int *slack_ids, int nslack, const double *slack_weights,
                        const int *pv, int npv, const int *pq, int npq, const pf_options *opts, pf_plan **out) {
    if (!out || !colptr || !rowind || !ybus_ri || !bp_colptr || !bp_rowind || !bp_x || !bpp_colptr || !bpp_rowind ||
        !bpp_x || !slack_ids || !slack_weights || (npv && !pv) || (npq && !pq))
        return fail(-1, "pf_fdpf_plan_create: null argument");
    *out = nullptr;
    pf_plan *pl = new pf_plan();
    if (opts) pl->opt = *opts;
    pl->opt.precision = 0;  // the reference's fast-decoupled solves are FP64
    l2g::PlanOptions po;
    if (pl->opt.pivot_threshold > 0) po.pivot_threshold = pl->opt.pivot_threshold;
    po.order_trials = pl->opt.ordering == 1 ? 0 : (pl->opt.ordering == 2 ? 1 : 8);
    po.level_slack = level_slack_of(pl->opt);
    po.elem_bytes = pl->opt.precision ? 4 : 8;
    po.spread_clusters = pl->opt.placement != 2;
    int thr = pl->opt.threads;
    if (thr <= 0) {
        // factors in global memory, read through L1 by every CTA of an SM, and several small
        // CTAs per SM to overlap the latency of the substitution phases: up to 8 while the solve
        // vectors stay within about 100 KB of shared memory per SM, else 4 CTAs of 128 threads,
        // or 2 of 256 for systems above 4000 unknowns (measured on 118- to 6515-bus grids)
        if (pl->opt.lu_placement == 1) {
            thr = 512;
        } else {
            const long long m_max = std::max<long long>(npv + nslack - 1 + npq, npq);
            const long long per = (m_max + 1) * 8 + 4096;
            int ctas = (int)std::min<long long>(8, (100 << 10) / per);
            thr = 128;
            if (ctas < 4) {
                ctas = m_max <= 4000 ? 4 : 2;
                thr = m_max <= 4000 ? 128 : 256;
            }
            if (pl->opt.max_ctas_per_sm <= 0) pl->opt.max_ctas_per_sm = ctas;
            if (pl->opt.lu_placement == 0) pl->opt.lu_placement = 2;
        }
    }
    thr = std::max(32, std::min(512, (thr / 32) * 32));
    po.threads = pl->threads = thr;
    po.fuse_forward = true;
    std::string msg;
    int rc;
    try {
        rc = l2g::build_fdpf_plan(pl->P, n, colptr, rowind, reinterpret_cast<const cplx *>(ybus_ri),
                                  l2g::RealCsc{bp_colptr, bp_rowind, bp_x}, l2g::RealCsc{bpp_colptr, bpp_rowind, bpp_x},
                                  slack_ids, nslack, slack_weights, pv, npv, pq, npq, po, msg);
    } catch (const std::exception &ex) {
        rc = -1;
        msg = std::string("pf_fdpf_plan_create: ") + ex.what();
    }
    if (rc != 0) {
        delete pl;
        return fail(rc, msg);
    }
    return finish_plan(pl, out);
}

void pf_plan_destroy(pf_plan *plan) {
    if (!plan) return;
    release(plan);
    delete plan;
}

int pf_plan_info_get(const pf_plan *pl, pf_plan_info *info) {
    if (!pl || !info) return fail(-1, "pf_plan_info_get: null argument");
    const l2g::Plan &P = pl->P;
    info->n = P.n;
    info->m = P.m;
    info->nnz_ybus = P.nnzY;
    info->nnz_j = (int)P.Ji.size();
    info->nnz_lu = P.nnzLU;
    info->levels_refactor = P.levels_refactor;
    info->levels_forward = P.levels_fwd;
    info->levels_backward = P.levels_bwd;
    info->groups_refactor = P.factor.nphases();
    info->groups_forward = P.forward.nphases();
    info->groups_backward = P.backward.nphases();
    info->flops_refactor = P.flops_refactor;
    if (P.fdpf) {
        // the two decoupled systems together (nothing is refactorised)
        info->nnz_j = (int)(P.sub[0].Ji.size() + P.sub[1].Ji.size());
        info->nnz_lu = P.sub[0].nnzLU + P.sub[1].nnzLU;
        info->levels_refactor = info->groups_refactor = 0;
        info->levels_forward = P.sub[0].levels_fwd + P.sub[1].levels_fwd;
        info->levels_backward = P.sub[0].levels_bwd + P.sub[1].levels_bwd;
        info->groups_forward = P.sub[0].forward.nphases() + P.sub[1].forward.nphases();
        info->groups_backward = P.sub[0].backward.nphases() + P.sub[1].backward.nphases();
        info->flops_refactor = 0;
    }
    info->precision = pl->precision;
    info->threads = pl->threads;
    info->lu_in_shared = pl->lu_in_smem ? 1 : 0;
    info->ctas_per_sm = pl->ctas_per_sm;
    info->grid = pl->grid;
    info->slab_bytes = (long long)pl->slab;
    info->shared_bytes = (long long)pl->smem;
    const bool packed = pl->lu_in_smem && !P.fdpf;
    info->smem_wavefronts_factor = packed ? l2g::smem_wavefronts(P, P.factor) : 0;
    info->smem_wavefronts_backward = packed ? l2g::smem_wavefronts(P, P.backward) : 0;
    info->smem_wavefronts_forward = packed ? l2g::smem_wavefronts(P, P.forward) : 0;
    info->tail_k = P.tail_k;
    return 0;
}

int pf_set_ybus_values(pf_plan *pl, const double *ybus_ri) {
    if (!pl || !ybus_ri) return fail(-1, "pf_set_ybus_values: null argument");
    l2g::Plan &P = pl->P;
    const cplx *y = reinterpret_cast<const cplx *>(ybus_ri);
    for (int p = 0; p < P.nnzY; ++p) {
        P.Yx[p] = y[p];
        P.Rx[P.csr_of_csc[p]] = y[p];
    }
    std::vector<double> rx(2 * (size_t)P.nnzY);
    for (int i = 0; i < P.nnzY; ++i) {
        rx[2 * i] = P.Rx[i].real();
        rx[2 * i + 1] = P.Rx[i].imag();
    }
    cudaError_t e = cudaMemcpy(const_cast<double2 *>(pl->dp.Rx), rx.data(), rx.size() * sizeof(double),
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "pf_set_ybus_values");
    compute_bridges(pl);
    return 0;
}

int pf_solve(pf_plan *pl, const double *V0_ri, const double *Sbus_ri, int max_iter, double tol, double *V_out_ri,
             int *converged, int *iters, int *err) {
    if (!pl || !V0_ri || !Sbus_ri || !V_out_ri) return fail(-1, "pf_solve: null argument");
    double t0 = now();
    std::vector<int> empty, jf{0}, jc{1};
    std::vector<cplx> ev;
    int it = 0, er = 0;
    int rc = run_batch(pl, 1, reinterpret_cast<const cplx *>(V0_ri), 0, reinterpret_cast<const cplx *>(Sbus_ri), 0,
                       empty, empty, ev, jf, jc, 0, max_iter, tol, reinterpret_cast<cplx *>(V_out_ri), &it, &er,
                       true);
    if (rc) return rc;
    pl->haveJ = it > 0;
    if (iters) *iters = it;
    if (err) *err = er;
    if (converged) *converged = er == 0;
    pl->timers[0] = now() - t0;
    pl->timers[1] = 0.0;
    return 0;
}

int pf_get_J(pf_plan *pl, int *m, int *Jp, int *Ji, double *Jx) {
    if (!pl) return fail(-1, "pf_get_J: null argument");
    if (pl->P.dc) return fail(-1, "pf_get_J: a DC plan has no Jacobian");
    if (pl->P.fdpf) return fail(-1, "pf_get_J: a fast-decoupled plan has no Jacobian");
    const l2g::Plan &P = pl->P;
    if (m) *m = P.m;
    if (Jp) std::memcpy(Jp, P.Jp.data(), P.Jp.size() * sizeof(int));
    if (Ji) std::memcpy(Ji, P.Ji.data(), P.Ji.size() * sizeof(int));
    if (Jx) {
        if (!pl->haveJ) return fail(-1, "pf_get_J: no iteration has been run yet");
        std::memcpy(Jx, pl->lastJ.data(), pl->lastJ.size() * sizeof(double));
    }
    return (int)P.Ji.size();
}

int pf_n1_prepare(pf_plan *pl, int ncases, const int *case_ptr, const int *coef_row, const int *coef_col,
                  const double *coef_val_ri, int *solvable, int *ovr_ptr, int *ovr_pos, double *ovr_val_ri, int cap) {
    if (!pl || ncases < 0 || !case_ptr || !solvable || !ovr_ptr) return fail(-1, "pf_n1_prepare: null argument");
    const cplx *cv = reinterpret_cast<const cplx *>(coef_val_ri);
    // per case, in parallel over contiguous parts of the cases: the overrides (status -1: a
    // coefficient outside the pattern, -2: more than kMaxOverrides entries, 0: islanded,
    // 1: solvable); then, in case order, the outputs and the first error, as a serial pass would
    struct Part {
        std::vector<int> status, first, pos;
        std::vector<cplx> val;
    };
    HostPool &pool = HostPool::get();
    const int nt = ncases >= 256 ? pool.threads() : 1;
    std::vector<Part> parts(nt);
    pool.run(nt, [&](int t, int nparts) {
        int lo, hi;
        part_range(ncases, t, nparts, lo, hi);
        Part &pt = parts[t];
        std::vector<int> opos;
        std::vector<cplx> oval;
        for (int c = lo; c < hi; ++c) {
            int st;
            if (case_overrides(pl->P, case_ptr[c], case_ptr[c + 1], coef_row, coef_col, cv, opos, oval) != 0)
                st = -1;
            else if ((int)opos.size() > l2g::kMaxOverrides)
                st = -2;
            else
                st = case_connected(pl, opos, oval) ? 1 : 0;
            pt.status.push_back(st);
            pt.first.push_back((int)pt.pos.size());
            if (st == 1) {
                pt.pos.insert(pt.pos.end(), opos.begin(), opos.end());
                pt.val.insert(pt.val.end(), oval.begin(), oval.end());
            }
            if (st < 0) break;  // the serial pass stops at this case
        }
        pt.first.push_back((int)pt.pos.size());
    });
    int w = 0, ns = 0;
    ovr_ptr[0] = 0;
    for (int t = 0; t < nt; ++t) {
        const Part &pt = parts[t];
        int lo, hi;
        part_range(ncases, t, nt, lo, hi);
        for (int i = 0; i < (int)pt.status.size(); ++i) {
            const int c = lo + i, st = pt.status[i];
            if (st == -1)
                return fail(-1, "pf_n1_prepare: case " + std::to_string(c) +
                                    " removes a coefficient that is not in the Ybus pattern");
            if (st == -2)
                return fail(-1, "pf_n1_prepare: case " + std::to_string(c) + " changes more than 32 Ybus entries");
            solvable[c] = st;
            if (!st) continue;
            const int k0 = pt.first[i], k1 = pt.first[i + 1];
            if (w + (k1 - k0) > cap) return -3;
            for (int k = k0; k < k1; ++k) {
                if (ovr_pos) ovr_pos[w] = pt.pos[k];
                if (ovr_val_ri) {
                    ovr_val_ri[2 * w] = pt.val[k].real();
                    ovr_val_ri[2 * w + 1] = pt.val[k].imag();
                }
                ++w;
            }
            ++ns;
            ovr_ptr[ns] = w;
        }
    }
    return w;
}

int pf_n1_order(const pf_plan *pl, int ninst, const int *ovr_ptr, const int *ovr_pos, const double *ovr_val_ri,
                const double *V0_ri, int *order) {
    if (!pl || ninst < 0 || !ovr_ptr || (ninst > 0 && (!ovr_pos || !ovr_val_ri)) || !V0_ri || !order)
        return fail(-1, "pf_n1_order: null argument");
    const l2g::Plan &P = pl->P;
    const cplx *V = reinterpret_cast<const cplx *>(V0_ri);
    const cplx *ov = reinterpret_cast<const cplx *>(ovr_val_ri);
    // score: max over the changed rows r of |dS_r|^2 (the squares rank as the magnitudes do),
    // dS_r = V_r conj(sum over the instance's changed entries (r, c) of dY V_c), at V0
    std::vector<double> score(ninst, 0.0);
    std::vector<char> bad(ninst, 0);
    HostPool &pool = HostPool::get();
    const int nt = ninst >= 256 ? pool.threads() : 1;
    pool.run(nt, [&](int t, int nparts) {
        int lo, hi;
        part_range(ninst, t, nparts, lo, hi);
        std::vector<std::pair<int, cplx>> rowsum;
        for (int i = lo; i < hi; ++i) {
            rowsum.clear();
            for (int k = ovr_ptr[i]; k < ovr_ptr[i + 1]; ++k) {
                const int p = ovr_pos[k];
                if (p < 0 || p >= P.nnzY) {
                    bad[i] = 1;
                    break;
                }
                const int r = P.Rrow[p], c = P.Rj[p];
                const cplx dI = (ov[k] - P.Rx[p]) * V[c];
                bool found = false;
                for (auto &e : rowsum)
                    if (e.first == r) {
                        e.second += dI;
                        found = true;
                    }
                if (!found) rowsum.push_back({r, dI});
            }
            double s = 0.0;
            for (auto &e : rowsum) s = std::max(s, std::norm(V[e.first] * std::conj(e.second)));
            score[i] = s;
        }
    });
    for (int i = 0; i < ninst; ++i)
        if (bad[i]) return fail(-1, "pf_n1_order: override position out of range");
    for (int i = 0; i < ninst; ++i) order[i] = i;
    std::stable_sort(order, order + ninst, [&](int a, int b) { return score[a] > score[b]; });
    return 0;
}

int pf_batch_n1(pf_plan *pl, int ncases, const int *case_ptr, const int *coef_row, const int *coef_col,
                const double *coef_val_ri, const double *V0_ri, const double *Sbus_ri, int max_iter, double tol,
                double *V_out_ri, int *converged, int *iters, int *errs) {
    if (!pl || ncases < 0 || !case_ptr || !V0_ri || !Sbus_ri || !V_out_ri || !converged || !iters || !errs)
        return fail(-1, "pf_batch_n1: null argument");
    double t0 = now();
    const int n = pl->P.n;
    std::vector<int> solv(ncases), optr(ncases + 1);
    int total = case_ptr[ncases] - case_ptr[0];
    std::vector<int> opos(std::max(total, 1));
    std::vector<cplx> oval(std::max(total, 1));
    int w = pf_n1_prepare(pl, ncases, case_ptr, coef_row, coef_col, coef_val_ri, solv.data(), optr.data(),
                          opos.data(), reinterpret_cast<double *>(oval.data()), (int)opos.size());
    if (w < 0) return w == -3 ? fail(-1, "pf_batch_n1: internal override buffer too small") : w;
    std::vector<int> idx;
    for (int c = 0; c < ncases; ++c)
        if (solv[c]) idx.push_back(c);
    const int ns = (int)idx.size();
    optr.resize(ns + 1);
    opos.resize(std::max(w, 1));
    oval.resize(std::max(w, 1));
    // jobs hardest first (largest power mismatch of the outage at V0): long instances start
    // early instead of extending the end of the launch; the results do not depend on the order
    std::vector<int> jf(ns), jc(ns, 1);
    {
        const int rc = pf_n1_order(pl, ns, optr.data(), opos.data(), reinterpret_cast<const double *>(oval.data()),
                                   V0_ri, jf.data());
        if (rc) return rc;
    }
    std::vector<int> it(std::max(ns, 1)), er(std::max(ns, 1));
    double t1 = now();
    cplx *Vo = reinterpret_cast<cplx *>(V_out_ri);
    // voltage rows straight into the caller's array when it is pinned and mapped into the device
    // address space: each instance's row is written (over the host link) as it finishes, the
    // islanded rows are zeroed on the host while the kernel runs, and nothing is copied after it
    {
        cudaPointerAttributes at{};
        const bool mapped = cudaPointerGetAttributes(&at, V_out_ri) == cudaSuccess &&
                            at.type == cudaMemoryTypeHost && at.devicePointer != nullptr;
        if (!mapped) cudaGetLastError();  // pageable memory: not an error
        if (mapped && ns > 0) {
            cudaError_t e = pl->casemap.ensure((size_t)ns * sizeof(int));
            if (e != cudaSuccess) return cuda_fail(e, "pf_batch_n1: alloc");
            e = cudaMemcpy(pl->casemap.p, idx.data(), (size_t)ns * sizeof(int), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return cuda_fail(e, "pf_batch_n1: upload");
            const std::function<void()> zero_islanded = [&]() {
                for (int c = 0; c < ncases; ++c)
                    if (!solv[c]) std::memset(Vo + (size_t)c * n, 0, (size_t)n * sizeof(cplx));
            };
            RowsOut ro;
            ro.vout = static_cast<double2 *>(at.devicePointer);
            ro.rows = static_cast<const int *>(pl->casemap.p);
            ro.during = &zero_islanded;
            int rc = run_batch(pl, ns, reinterpret_cast<const cplx *>(V0_ri), 0,
                               reinterpret_cast<const cplx *>(Sbus_ri), 0, optr, opos, oval, jf, jc, 0, max_iter,
                               tol, nullptr, it.data(), er.data(), false, nullptr, &ro);
            if (rc) return rc;
            for (int c = 0; c < ncases; ++c) {
                converged[c] = 0;
                iters[c] = 0;
                errs[c] = 1;  // SingularMatrix: islanded, not computed
            }
            for (int i = 0; i < ns; ++i) {
                const int c = idx[i];
                iters[c] = it[i];
                errs[c] = er[i];
                converged[c] = er[i] == 0;
            }
            pl->timers[0] = now() - t0;
            pl->timers[1] = t1 - t0;
            return 0;
        }
    }
    // otherwise: result rows in case order on the device, then one copy into the caller's array,
    // on the copy stream: issued as soon as the rows are final, so the copy overlaps the FP64
    // re-run of the instances that failed in the mixed form; their rows follow once it is done
    cudaStream_t cs = pl->copy_stream;
    std::vector<int> map(ncases, -1);
    for (int i = 0; i < ns; ++i) map[idx[i]] = i;
    std::vector<char> rerun_rows;
    const std::function<int(const std::vector<char> &)> settled = [&](const std::vector<char> &again) -> int {
        std::vector<int> m1 = map;
        for (int c = 0; c < ncases; ++c)
            if (m1[c] >= 0 && again[m1[c]]) m1[c] = -1;  // zero for now, copied after the re-run
        rerun_rows = again;
        cudaError_t e;
        if ((e = pl->casemap.ensure((size_t)std::max(ncases, 1) * sizeof(int))) != cudaSuccess)
            return cuda_fail(e, "pf_batch_n1: alloc");
        if ((e = pl->Vcase.ensure((size_t)std::max(ncases, 1) * n * sizeof(cplx))) != cudaSuccess)
            return cuda_fail(e, "pf_batch_n1: alloc");
        if ((e = cudaMemcpyAsync(pl->casemap.p, m1.data(), (size_t)ncases * sizeof(int), cudaMemcpyHostToDevice,
                                 cs)) != cudaSuccess)
            return cuda_fail(e, "pf_batch_n1: upload");
        if ((e = cudaStreamSynchronize(cs)) != cudaSuccess) return cuda_fail(e, "pf_batch_n1: upload");
        if ((e = l2g::launch_scatter_case_rows(static_cast<const double2 *>(pl->Vout.p),
                                               static_cast<const int *>(pl->errs.p),
                                               static_cast<const int *>(pl->casemap.p), ncases, n,
                                               static_cast<double2 *>(pl->Vcase.p), pl->num_sms, cs)) != cudaSuccess)
            return cuda_fail(e, "pf_batch_n1: scatter");
        if ((e = cudaMemcpyAsync(Vo, pl->Vcase.p, (size_t)ncases * n * sizeof(cplx), cudaMemcpyDeviceToHost, cs)) !=
            cudaSuccess)
            return cuda_fail(e, "pf_batch_n1: download");
        return 0;
    };
    if (ns > 0) {
        int rc = run_batch(pl, ns, reinterpret_cast<const cplx *>(V0_ri), 0, reinterpret_cast<const cplx *>(Sbus_ri),
                           0, optr, opos, oval, jf, jc, 0, max_iter, tol, nullptr, it.data(), er.data(), false,
                           &settled);
        if (rc) {
            cudaStreamSynchronize(cs);
            return rc;
        }
        // rows of re-run instances that converged in FP64 (the others stay zero)
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < ns && e == cudaSuccess; ++i)
            if (rerun_rows[i] && er[i] == 0)
                e = cudaMemcpyAsync(Vo + (size_t)idx[i] * n, static_cast<const cplx *>(pl->Vout.p) + (size_t)i * n,
                                    (size_t)n * sizeof(cplx), cudaMemcpyDeviceToHost, cs);
        if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
        if (e != cudaSuccess) return cuda_fail(e, "pf_batch_n1: download");
    } else {
        cudaStream_t st = pl->stream;
        cudaError_t e;
        if ((e = pl->casemap.ensure((size_t)std::max(ncases, 1) * sizeof(int))) != cudaSuccess)
            return cuda_fail(e, "pf_batch_n1: alloc");
        if ((e = pl->Vcase.ensure((size_t)std::max(ncases, 1) * n * sizeof(cplx))) != cudaSuccess)
            return cuda_fail(e, "pf_batch_n1: alloc");
        if (ns == 0 && (e = pl->errs.ensure(sizeof(int))) != cudaSuccess) return cuda_fail(e, "pf_batch_n1: alloc");
        if (ns == 0 && (e = pl->Vout.ensure(sizeof(cplx))) != cudaSuccess) return cuda_fail(e, "pf_batch_n1: alloc");
        if ((e = cudaMemcpyAsync(pl->casemap.p, map.data(), (size_t)ncases * sizeof(int), cudaMemcpyHostToDevice,
                                 st)) != cudaSuccess)
            return cuda_fail(e, "pf_batch_n1: upload");
        if ((e = l2g::launch_scatter_case_rows(static_cast<const double2 *>(pl->Vout.p),
                                               static_cast<const int *>(pl->errs.p),
                                               static_cast<const int *>(pl->casemap.p), ncases, n,
                                               static_cast<double2 *>(pl->Vcase.p), pl->num_sms, st)) != cudaSuccess)
            return cuda_fail(e, "pf_batch_n1: scatter");
        if ((e = cudaMemcpyAsync(Vo, pl->Vcase.p, (size_t)ncases * n * sizeof(cplx), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess)
            return cuda_fail(e, "pf_batch_n1: download");
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "pf_batch_n1: download");
    }
    for (int c = 0; c < ncases; ++c) {
        converged[c] = 0;
        iters[c] = 0;
        errs[c] = 1;  // SingularMatrix: islanded, not computed
    }
    for (int i = 0; i < ns; ++i) {
        int c = idx[i];
        iters[c] = it[i];
        errs[c] = er[i];
        converged[c] = er[i] == 0;
    }
    pl->timers[0] = now() - t0;
    pl->timers[1] = t1 - t0;
    return 0;
}

int pf_batch_ts(pf_plan *pl, int nsteps, const double *Sbus_ri, const double *V0_ri, int nchunks, int max_iter,
                double tol, double *V_out_ri, int *converged, int *iters, int *errs, int *status) {
    if (!pl || nsteps < 0 || !Sbus_ri || !V0_ri || !V_out_ri || !converged || !iters || !errs)
        return fail(-1, "pf_batch_ts: null argument");
    double t0 = now();
    const int n = pl->P.n;
    if (nchunks <= 0) nchunks = pl->grid;
    nchunks = std::max(1, std::min(nchunks, std::max(nsteps, 1)));
    std::vector<int> jf, jc;
    for (int c = 0; c < nchunks; ++c) {
        int a = (int)((long long)nsteps * c / nchunks), b = (int)((long long)nsteps * (c + 1) / nchunks);
        if (b > a) {
            jf.push_back(a);
            jc.push_back(b - a);
        }
    }
    std::vector<int> empty;
    std::vector<cplx> ev;
    int rc = 0;
    // a pinned, device-mapped output takes each step's row straight from the kernel (as in
    // pf_batch_n1); otherwise the rows are copied after the kernel
    cudaPointerAttributes at{};
    const bool mapped = cudaPointerGetAttributes(&at, V_out_ri) == cudaSuccess && at.type == cudaMemoryTypeHost &&
                        at.devicePointer != nullptr;
    if (!mapped) cudaGetLastError();
    RowsOut ro;
    ro.vout = mapped ? static_cast<double2 *>(at.devicePointer) : nullptr;
    if (nsteps > 0)
        rc = run_batch(pl, nsteps, reinterpret_cast<const cplx *>(V0_ri), 0, reinterpret_cast<const cplx *>(Sbus_ri), n,
                       empty, empty, ev, jf, jc, 1, max_iter, tol,
                       mapped ? nullptr : reinterpret_cast<cplx *>(V_out_ri), iters, errs, false, nullptr,
                       mapped ? &ro : nullptr);
    if (rc) return rc;
    int first_bad = nsteps;
    for (int s = 0; s < nsteps; ++s)
        if (errs[s] != 0) {
            first_bad = s;
            break;
        }
    cplx *Vo = reinterpret_cast<cplx *>(V_out_ri);
    for (int s = 0; s < nsteps; ++s) {
        converged[s] = s < first_bad;
        if (s >= first_bad) {
            std::fill(Vo + (size_t)s * n, Vo + (size_t)(s + 1) * n, cplx(0.0, 0.0));
            if (s > first_bad) {
                iters[s] = 0;
                errs[s] = 8;
            }
        }
    }
    if (status) *status = first_bad == nsteps ? 1 : 0;
    pl->timers[0] = now() - t0;
    pl->timers[1] = 0.0;
    return 0;
}


static int batch_device_impl(pf_plan *pl, const pf_device_batch *b, void *stream, unsigned long long *cycles) {
    l2g::BatchArgs a = l2g::device_args(b);
    a.phase_cycles = cycles;
    return launch(pl, a, pl->precision, static_cast<cudaStream_t>(stream));
}


int pf_batch_device_scratch(pf_plan *plan, const pf_device_batch *batch, void *scratch, long long scratch_bytes,
                            void *stream) {
    if (scratch_bytes <= 0) return fail(-1, "pf_batch_device_scratch: scratch too small");
    return l2g::batch_device_with_scratch(plan, batch, stream, scratch, (size_t)scratch_bytes, false);
}

long long pf_scratch_bytes(const pf_plan *plan, int ctas) {
    if (!plan || ctas <= 0) return fail(-1, "pf_scratch_bytes: invalid argument");
    const int c = std::min(ctas, plan->grid);
    return 256 + (long long)plan->slab * c;
}

int pf_batch_device(pf_plan *pl, const pf_device_batch *b, void *stream) {
    if (!pl || !b) return fail(-1, "pf_batch_device: null argument");
    if (int rc = check_plan_device(pl->device, "pf_batch_device")) return rc;
    return batch_device_impl(pl, b, stream, nullptr);
}

int pf_batch_device_phase_trace(pf_plan *pl, const pf_device_batch *b, void *stream, double *out, int cap) {
    if (!pl || !b || !out || cap <= 0) return fail(-1, "pf_batch_device_phase_trace: null argument");
    cudaError_t e = pl->cycles.ensure((size_t)cap * sizeof(unsigned long long));
    if (e != cudaSuccess) return cuda_fail(e, "pf_batch_device_phase_trace: alloc");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    e = cudaMemsetAsync(pl->cycles.p, 0, (size_t)cap * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_fail(e, "pf_batch_device_phase_trace: memset");
    l2g::BatchArgs a = l2g::device_args(b);
    a.trace = static_cast<unsigned long long *>(pl->cycles.p);
    a.trace_cap = cap;
    int rc = launch(pl, a, pl->precision, st);
    if (rc) return rc;
    std::vector<unsigned long long> h(cap);
    e = cudaMemcpyAsync(h.data(), pl->cycles.p, (size_t)cap * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "pf_batch_device_phase_trace: download");
    int n = 0;
    while (n < cap && h[n] != 0) ++n;
    for (int i = 0; i < n; ++i) out[i] = i == 0 ? 0.0 : (double)(h[i] - h[0]);
    return n;
}

int pf_batch_device_phase_cycles(pf_plan *pl, const pf_device_batch *b, void *stream, double *out) {
    if (!pl || !b || !out) return fail(-1, "pf_batch_device_phase_cycles: null argument");
    const size_t slots = (size_t)pl->grid * l2g::kPhaseSlots;
    cudaError_t e = pl->cycles.ensure(slots * sizeof(unsigned long long));
    if (e != cudaSuccess) return cuda_fail(e, "pf_batch_device_phase_cycles: alloc");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    e = cudaMemsetAsync(pl->cycles.p, 0, slots * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_fail(e, "pf_batch_device_phase_cycles: memset");
    int rc = batch_device_impl(pl, b, stream, static_cast<unsigned long long *>(pl->cycles.p));
    if (rc) return rc;
    std::vector<unsigned long long> h(slots);
    e = cudaMemcpyAsync(h.data(), pl->cycles.p, slots * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "pf_batch_device_phase_cycles: download");
    for (int i = 0; i < l2g::kPhaseSlots; ++i) {
        double acc = 0.0;
        for (int b2 = 0; b2 < pl->grid; ++b2) acc += (double)h[(size_t)b2 * l2g::kPhaseSlots + i];
        out[i] = acc;
    }
    return 0;
}

int pf_timers(const pf_plan *pl, double *out, int nout) {
    if (!pl || !out) return fail(-1, "pf_timers: null argument");
    for (int i = 0; i < nout && i < 6; ++i) out[i] = pl->timers[i];
    return 0;
}

int pf_host_jacobian_pattern(int n, const int *colptr, const int *rowind, const double *ybus_ri,
                             const int *slack_ids, int nslack, const double *slack_weights, const int *pv, int npv,
                             const int *pq, int npq, int distributed, int *m, int *Jp, int *Ji) {
    if (!colptr || !rowind || !ybus_ri || !slack_ids || !slack_weights) return fail(-1, "null argument");
    l2g::Plan P;
    l2g::PlanOptions po;
    std::string msg;
    std::vector<cplx> V0(n, cplx(1.0, 0.0)), S(n, cplx(0.0, 0.0));
    int rc = l2g::build_plan(P, n, colptr, rowind, reinterpret_cast<const cplx *>(ybus_ri), V0.data(), S.data(),
                             slack_ids, nslack, slack_weights, pv, npv, pq, npq, distributed != 0, po, msg);
    // a flat start may give a singular first Jacobian; the pattern is still valid then
    if (rc != 0 && P.Jp.empty()) return fail(rc, msg);
    if (m) *m = P.m;
    if (Jp) std::memcpy(Jp, P.Jp.data(), P.Jp.size() * sizeof(int));
    if (Ji) std::memcpy(Ji, P.Ji.data(), P.Ji.size() * sizeof(int));
    return (int)P.Ji.size();
}

int pf_host_schedule_solve(int n, const int *colptr, const int *rowind, const double *ybus_ri, const double *V0_ri,
                           const double *V_ri, const int *slack_ids, int nslack, const double *slack_weights,
                           const int *pv, int npv, const int *pq, int npq, int distributed, const double *b,
                           double *x, pf_plan_info *info) {
    if (!colptr || !rowind || !ybus_ri || !V0_ri || !V_ri || !b || !x) return fail(-1, "null argument");
    l2g::Plan P;
    l2g::PlanOptions po;
    std::string msg;
    std::vector<cplx> S(n, cplx(0.0, 0.0));
    int rc = l2g::build_plan(P, n, colptr, rowind, reinterpret_cast<const cplx *>(ybus_ri),
                             reinterpret_cast<const cplx *>(V0_ri), S.data(), slack_ids, nslack, slack_weights, pv,
                             npv, pq, npq, distributed != 0, po, msg);
    if (rc != 0) return fail(rc, msg);
    const int m = P.m;
    std::vector<double> Jx;
    l2g::host_jacobian(P, P.Yx.data(), reinterpret_cast<const cplx *>(V_ri), Jx);
    // scatter J into the LU layout exactly as the device fill does
    std::vector<double> lu(P.nnzLU, 0.0);
    std::vector<char> seen(P.nnzLU, 0);
    for (int d = 0; d < P.nnzY; ++d)
        for (int k = 0; k < 4; ++k) {
            int t = P.ytarget[4 * (size_t)d + k], j = P.yjpos[4 * (size_t)d + k];
            if (t >= 0) { lu[t] = Jx[j]; seen[t] = 1; }
        }
    for (size_t i = 0; i < P.cpos.size(); ++i) { lu[P.cpos[i]] = P.cval[i]; seen[P.cpos[i]] = 1; }
    for (int p : P.fillpos) { lu[p] = 0.0; seen[p] = 1; }
    for (int p = 0; p < P.nnzLU; ++p)
        if (!seen[p]) return fail(-1, "schedule check: an LU position is never written by the fill");
    // permuted right-hand side, as the device mismatch writes it
    std::vector<double> xs(m, 0.0);
    for (int f = 0; f < m; ++f) xs[P.pinv[f]] = b[f];
    // the device's phase programs, one operation after the other (a phase's operations are
    // independent, so any order gives the device's result)
    auto run = [&](const l2g::Plan::Program &pr) {
        for (int o = 0; o < pr.nops(); ++o) {
            const int X = pr.ops[4 * o], Y = pr.ops[4 * o + 1], Z = pr.ops[4 * o + 2];
            const int W = pr.ops[4 * o + 3] & 0x0fffffff, kind = (unsigned)pr.ops[4 * o + 3] >> 28;
            switch (kind) {
                case 0: lu[X] -= lu[Y] * (lu[Z] / lu[W]); break;
                case 2: xs[X] -= lu[Y] * xs[Z] / lu[W]; break;
                default: break;
            }
        }
    };
    // the same programs in the packed form of the shared-memory layout, one index space
    std::vector<double> s0;
    if (l2g::compact_fits(P)) {
        const int L = l2g::compact_lu_offset(m);
        s0.assign((size_t)L + P.nnzLU, 0.0);
        for (int k = 0; k < m; ++k) s0[k] = xs[k];
        for (int p = 0; p < P.nnzLU; ++p) s0[(size_t)L + p] = lu[p];
    }
    auto run_packed = [&](const l2g::Plan::Program &pr) {
        std::vector<unsigned> c;
        l2g::compact_ops(pr, m, c);
        for (size_t o = 0; o < c.size(); o += 2) {
            const unsigned X = c[o] & 0xffffu, Y = c[o] >> 16, Z = c[o + 1] & 0xffffu, W = c[o + 1] >> 16;
            if (X == (unsigned)m) continue;  // empty slot (scratch)
            s0[X] -= s0[Y] * (s0[Z] / s0[W]);
        }
    };
    auto scale = [&](std::vector<double> &v, const double *u) {
        for (int k = 0; k < m; ++k) v[k] = v[k] / u[P.dpos[k]];
    };
    // the dense tail, as the kernel runs it: after the factor program the block is gathered and
    // factorised without pivoting (unit lower L), its pivots written back to the LU diagonal; the
    // block's forward substitution follows the factor (or forward) program, its backward
    // substitution (undivided values, as the backward program) precedes the backward program
    const int tk = P.tail_k, tc = P.tail_ct;
    std::vector<double> D;
    auto tail_factor = [&]() {
        if (tk == 0) return;
        D.assign((size_t)tk * tk, 0.0);
        for (size_t e = 0; e < D.size(); ++e)
            if (P.tail_map[e] >= 0) D[e] = lu[P.tail_map[e]];
        for (int c = 0; c < tk; ++c) {
            const double piv = D[(size_t)c * tk + c];
            for (int i = c + 1; i < tk; ++i) {
                const double l = D[(size_t)i * tk + c] / piv;
                D[(size_t)i * tk + c] = l;
                for (int j = c + 1; j < tk; ++j) D[(size_t)i * tk + j] -= l * D[(size_t)c * tk + j];
            }
        }
        for (int c = 0; c < tk; ++c) lu[P.dpos[tc + c]] = D[(size_t)c * tk + c];
    };
    auto tail_forward = [&](std::vector<double> &v) {
        for (int c = 0; c < tk; ++c)
            for (int i = c + 1; i < tk; ++i) v[tc + i] -= D[(size_t)i * tk + c] * v[tc + c];
    };
    auto tail_backward = [&](std::vector<double> &v) {
        for (int c = tk - 1; c >= 0; --c) {
            const double w = v[tc + c] / D[(size_t)c * tk + c];
            for (int i = 0; i < c; ++i) v[tc + i] -= D[(size_t)i * tk + c] * w;
        }
    };
    const std::vector<double> lu0 = lu, xs0 = xs;
    // the bank-conflict placement of the packed programs gives the same bits: every written
    // value keeps its thread and the order of its operations.  Checked for the placement of this
    // plan (4-byte words), for the one built for 8-byte words (FP64) and for the spread clusters.
    {
        std::vector<double> la = lu, xa = xs, xf = xs;  // longest-first: factor + backward; forward
        std::swap(la, lu);
        std::swap(xa, xs);
        run(P.factor);
        run(P.backward);
        std::swap(xa, xs);
        std::swap(xf, xs);
        run(P.forward);  // on the factor just computed
        std::swap(xf, xs);
        std::swap(la, lu);
        // the same plan built for 8-byte words, and with the clusters spread over the slots
        l2g::Plan P8, Ps;
        const l2g::Plan *variants[3] = {&P, nullptr, nullptr};
        if (P.bank_lanes > 0) {
            l2g::Plan *Q[2] = {&P8, &Ps};
            for (int v = 0; v < 2; ++v) {
                l2g::PlanOptions pv2 = po;
                if (v == 0) pv2.elem_bytes = 8;
                else pv2.spread_clusters = true;
                std::string msg2;
                if (l2g::build_plan(*Q[v], n, colptr, rowind, reinterpret_cast<const cplx *>(ybus_ri),
                                    reinterpret_cast<const cplx *>(V0_ri), S.data(), slack_ids, nslack, slack_weights,
                                    pv, npv, pq, npq, distributed != 0, pv2, msg2) != 0 ||
                    Q[v]->factor.ops != P.factor.ops || Q[v]->backward.ops != P.backward.ops ||
                    Q[v]->forward.ops != P.forward.ops)
                    return fail(-1, "schedule check: a placement variant of the plan differs");
                variants[1 + v] = Q[v];
            }
        }
        for (const l2g::Plan *Q : variants) {
            if (!Q) continue;
            std::vector<double> lb = lu, xb = xs;
            auto run_banked = [&](const l2g::Plan::Program &pr) {
                const std::vector<int> &ops = pr.ops_banked.empty() ? pr.ops : pr.ops_banked;
                for (int o = 0; o < pr.nops(); ++o) {
                    const int X = ops[4 * o], Y = ops[4 * o + 1], Z = ops[4 * o + 2];
                    const int W = ops[4 * o + 3] & 0x0fffffff, kind = (unsigned)ops[4 * o + 3] >> 28;
                    if (kind == 0) lb[X] -= lb[Y] * (lb[Z] / lb[W]);
                    else if (kind == 2) xb[X] -= lb[Y] * xb[Z] / lb[W];
                }
            };
            run_banked(Q->factor);
            run_banked(Q->backward);
            for (int p = 0; p < P.nnzLU; ++p)
                if (lb[p] != la[p]) return fail(-1, "schedule check: bank-placed factor program disagrees");
            for (int k = 0; k < m; ++k)
                if (xb[k] != xa[k]) return fail(-1, "schedule check: bank-placed substitution programs disagree");
            xb = xs;
            run_banked(Q->forward);
            for (int k = 0; k < m; ++k)
                if (xb[k] != xf[k]) return fail(-1, "schedule check: bank-placed forward program disagrees");
        }
    }
    run(P.factor);
    tail_factor();
    tail_forward(xs);
    for (int k = 0; k < m; ++k)
        if (lu[P.dpos[k]] == 0.0) return fail(l2g::SolverReFactor, "schedule check: zero pivot");
    tail_backward(xs);
    run(P.backward);
    scale(xs, lu.data());
    // the instance-interleaved batch programs (groups per warp, chunk after chunk) give the same
    // bits: every written value sees its operations in the same order (plans without a dense
    // tail: the interleaved kernel runs those only)
    if (tk == 0) {
        std::vector<double> lt = lu0, xt = xs0;
        auto run_tile = [&](const l2g::Plan::Program &pr, std::vector<double> &v) {
            l2g::TileProgram tp;
            l2g::build_tile_program(pr, l2g::kTileWarps, l2g::kTileChunk, tp);
            for (size_t p = 0; p + 1 < tp.phase.size(); p += 2)
                for (int w = 0; w < l2g::kTileWarps; ++w)
                    for (int r = 0; r < tp.phase[p + 1]; ++r) {
                        const size_t c = (size_t)tp.phase[p] + (size_t)r * l2g::kTileWarps + w;
                        for (int q = 0; q < l2g::kTileChunk; ++q) {
                            const int *o = &tp.ops[4 * (c * l2g::kTileChunk + q)];
                            const int W = o[3] & 0x0fffffff, kind = (unsigned)o[3] >> 28;
                            if (kind == 0) lt[o[0]] -= lt[o[1]] * (lt[o[2]] / lt[W]);
                            else if (kind == 2) v[o[0]] -= lt[o[1]] * v[o[2]] / lt[W];
                        }
                    }
        };
        run_tile(P.factor, xt);
        run_tile(P.backward, xt);
        scale(xt, lt.data());
        for (int k = 0; k < m; ++k)
            if (xt[k] != xs[k]) return fail(-1, "schedule check: batch-interleaved programs disagree");
        std::vector<double> y3(m, 0.0);
        for (int f = 0; f < m; ++f) y3[P.pinv[f]] = b[f];
        run_tile(P.forward, y3);
        std::vector<double> y4(m, 0.0);
        for (int f = 0; f < m; ++f) y4[P.pinv[f]] = b[f];
        std::vector<double> lsave = lu;
        lu = lt;
        std::swap(xs, y4);
        run(P.forward);
        std::swap(xs, y4);
        lu = lsave;
        for (int k = 0; k < m; ++k)
            if (y3[k] != y4[k]) return fail(-1, "schedule check: batch-interleaved forward program disagrees");
    }
    if (!s0.empty() && tk == 0) {
        const int L = l2g::compact_lu_offset(m);
        run_packed(P.factor);
        run_packed(P.backward);
        std::vector<double> xc(s0.begin(), s0.begin() + m);
        scale(xc, s0.data() + L);
        double dmax = 0.0, amax = 0.0;
        for (int k = 0; k < m; ++k) {
            dmax = std::max(dmax, std::fabs(xc[k] - xs[k]));
            amax = std::max(amax, std::fabs(xs[k]));
        }
        if (dmax > 1e-9 * std::max(1.0, amax))
            return fail(-1, "schedule check: packed and unpacked programs disagree");
    }
    // the stand-alone forward program must agree with the fused one: solve L y = b again
    {
        std::vector<double> y2(m, 0.0), keep = xs;
        for (int f = 0; f < m; ++f) y2[P.pinv[f]] = b[f];
        xs = y2;
        run(P.forward);
        tail_forward(xs);
        tail_backward(xs);
        run(P.backward);
        scale(xs, lu.data());
        double dmax = 0.0, amax = 0.0;
        for (int k = 0; k < m; ++k) {
            dmax = std::max(dmax, std::fabs(xs[k] - keep[k]));
            amax = std::max(amax, std::fabs(keep[k]));
        }
        if (dmax > 1e-9 * std::max(1.0, amax))
            return fail(-1, "schedule check: fused and stand-alone forward substitutions disagree");
        xs = keep;
    }
    for (int v = 0; v < m; ++v) x[v] = xs[P.qinv[v]];
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->n = P.n;
        info->m = P.m;
        info->nnz_ybus = P.nnzY;
        info->nnz_j = (int)P.Ji.size();
        info->nnz_lu = P.nnzLU;
        info->levels_refactor = P.levels_refactor;
        info->levels_forward = P.levels_fwd;
        info->levels_backward = P.levels_bwd;
        info->groups_refactor = P.factor.nphases();
        info->groups_forward = P.forward.nphases();
        info->groups_backward = P.backward.nphases();
        info->flops_refactor = P.flops_refactor;
        // the packed layout's bank model, where the plan has one (FP32 element size here)
        info->smem_wavefronts_factor = l2g::smem_wavefronts(P, P.factor);
        info->smem_wavefronts_backward = l2g::smem_wavefronts(P, P.backward);
        info->smem_wavefronts_forward = l2g::smem_wavefronts(P, P.forward);
        info->tail_k = P.tail_k;
    }
    return 0;
}


int pf_multi_create(pf_plan *const *plans, const pf_device_batch *batches, int nseg, const int *job_seg,
                    const int *job_first, const int *job_count, int njobs, pf_multi **out) {
    if (!out || !plans || !batches || nseg <= 0 || njobs < 0 || (njobs > 0 && (!job_seg || !job_first || !job_count)))
        return fail(-1, "pf_multi_create: invalid argument");
    *out = nullptr;
    pf_multi *mp = new pf_multi();
    for (int i = 0; i < nseg; ++i) {
        pf_plan *pl = plans[i];
        if (!pl) {
            delete mp;
            return fail(-1, "pf_multi_create: null plan");
        }
        if (i == 0) {
            mp->device = pl->device;
            mp->precision = pl->precision;
            mp->refine = pl->refine;
            mp->lu_in_smem = pl->lu_in_smem;
            mp->num_sms = pl->num_sms;
        } else if (pl->device != mp->device || pl->precision != mp->precision || pl->refine != mp->refine ||
                   pl->lu_in_smem != mp->lu_in_smem) {
            delete mp;
            return fail(-1, "pf_multi_create: plans differ in device, precision, refinement or LU placement");
        }
        if (pl->P.dc || pl->P.fdpf) {
            delete mp;
            return fail(-1, "pf_multi_create: DC and fast-decoupled plans run one plan per launch");
        }
        mp->plans.push_back(pl);
        mp->threads = std::max(mp->threads, pl->threads);
        mp->smem = std::max(mp->smem, pl->smem);
        mp->slab = std::max(mp->slab, pl->slab);
    }
    int occ = l2g::nr_occupancy(mp->precision, mp->lu_in_smem, mp->refine, mp->threads, mp->smem);
    if (occ <= 0) {
        delete mp;
        return fail(-1, "pf_multi_create: the plans' largest layout cannot be launched");
    }
    mp->grid = std::max(1, std::min(mp->num_sms * occ, std::max(njobs, 1)));
    cudaError_t e;
    if ((e = mp->scratch.ensure(mp->slab * (size_t)mp->grid)) != cudaSuccess ||
        (e = mp->counter.ensure(256)) != cudaSuccess ||
        (e = mp->segs.ensure(sizeof(l2g::Segment) * (size_t)nseg)) != cudaSuccess) {
        for (DevBuf *b : {&mp->scratch, &mp->counter, &mp->segs}) b->release();
        delete mp;
        return cuda_fail(e, "pf_multi_create: allocation");
    }
    std::vector<l2g::Segment> host(nseg);
    for (int i = 0; i < nseg; ++i) {
        pf_plan *pl = plans[i];
        l2g::Segment &sg = host[i];
        sg.P = pl->dp;
        sg.A = l2g::device_args(&batches[i]);
        sg.A.scratch = static_cast<unsigned char *>(mp->scratch.p);
        sg.A.slab_bytes = (long long)mp->slab;
        sg.A.job_counter = nullptr;  // jobs come from the launch's list
        sg.A.lu_in_smem = mp->lu_in_smem ? 1 : 0;
        sg.A.refine = mp->refine ? 1 : 0;
        sg.A.refine_below = pl->opt.refine_threshold > 0 ? pl->opt.refine_threshold : 1e-3;
        sg.A.reuse_below = lu_reuse_below(pl, sg.A.refine_below);
    }
    e = cudaMemcpy(mp->segs.p, host.data(), sizeof(l2g::Segment) * (size_t)nseg, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        for (DevBuf *b : {&mp->scratch, &mp->counter, &mp->segs}) b->release();
        delete mp;
        return cuda_fail(e, "pf_multi_create: upload");
    }
    mp->seg0 = host[0];
    mp->M.segs = static_cast<const l2g::Segment *>(mp->segs.p);
    mp->M.job_seg = job_seg;
    mp->M.job_first = job_first;
    mp->M.job_count = job_count;
    mp->M.njobs = njobs;
    mp->M.job_counter = static_cast<int *>(mp->counter.p);
    *out = mp;
    return 0;
}

int pf_multi_launch(pf_multi *mp, void *stream) {
    if (!mp) return fail(-1, "pf_multi_launch: null argument");
    if (int rc = check_plan_device(mp->device, "pf_multi_launch")) return rc;
    if (mp->M.njobs <= 0) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(mp->counter.p, 0, sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(e, "pf_multi_launch: counter reset");
    l2g::BatchArgs a0 = mp->seg0.A;
    a0.phase_cycles = nullptr;
    a0.trace = nullptr;
    e = l2g::launch_nr_batch(mp->seg0.P, a0, mp->precision, mp->threads, mp->grid, mp->smem, st, mp->M);
    if (e != cudaSuccess) return cuda_fail(e, "pf_multi_launch: kernel");
    return 0;
}

int pf_multi_info(const pf_multi *mp, int *threads, int *grid, long long *shared_bytes, long long *scratch_bytes) {
    if (!mp) return fail(-1, "pf_multi_info: null argument");
    if (threads) *threads = mp->threads;
    if (grid) *grid = mp->grid;
    if (shared_bytes) *shared_bytes = (long long)mp->smem;
    if (scratch_bytes) *scratch_bytes = (long long)(mp->slab * (size_t)mp->grid);
    return 0;
}

void pf_multi_destroy(pf_multi *mp) {
    if (!mp) return;
    for (DevBuf *b : {&mp->scratch, &mp->counter, &mp->segs}) b->release();
    delete mp;
}


int pf_flows_device(const pf_branch_set *br, int n, int nrows, const double *V_ri, long long v_stride,
                    const int *map, const int *errs, const int *out_ptr, const int *out_ids, double *amps,
                    double *p_mw, void *stream) {
    if (!br || nrows < 0 || n <= 0 || br->nbr < 0 || (nrows > 0 && br->nbr > 0 && (!V_ri || !br->from || !br->to ||
                                                                                     !br->yff_ri || !br->yft_ri ||
                                                                                     !br->vn_kv_from)))
        return fail(-1, "pf_flows_device: invalid argument");
    if (out_ptr && !out_ids) return fail(-1, "pf_flows_device: out_ids missing");
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "pf_flows_device: device query");
    l2g::FlowArgs a{};
    a.V = reinterpret_cast<const double2 *>(V_ri);
    a.v_stride = v_stride;
    a.map = map;
    a.errs = errs;
    a.nrows = nrows;
    a.n = n;
    a.from = br->from;
    a.to = br->to;
    a.yff = reinterpret_cast<const double2 *>(br->yff_ri);
    a.yft = reinterpret_cast<const double2 *>(br->yft_ri);
    a.vn_kv_from = br->vn_kv_from;
    a.status = br->status;
    a.nbr = br->nbr;
    a.sn_mva = br->sn_mva;
    a.out_ptr = out_ptr;
    a.out_ids = out_ids;
    a.amps = amps;
    a.p_mw = p_mw;
    e = l2g::launch_branch_flows(a, sms, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "pf_flows_device: kernel");
    return 0;
}

int pf_flows_host(const pf_branch_set *br, int n, int nrows, const double *V_ri, const int *out_ptr,
                  const int *out_ids, double *amps, double *p_mw) {
    if (!br || nrows < 0 || n <= 0 || br->nbr < 0) return fail(-1, "pf_flows_host: invalid argument");
    const int nb = br->nbr;
    if (nrows == 0 || nb == 0) return 0;
    if (!V_ri || !br->from || !br->to || !br->yff_ri || !br->yft_ri || !br->vn_kv_from)
        return fail(-1, "pf_flows_host: null argument");
    for (int k = 0; k < nb; ++k)
        if (br->from[k] < 0 || br->from[k] >= n || br->to[k] < 0 || br->to[k] >= n)
            return fail(-1, "pf_flows_host: branch bus index out of range");
    int nout = 0;
    if (out_ptr) {
        if (!out_ids) return fail(-1, "pf_flows_host: out_ids missing");
        if (out_ptr[0] != 0) return fail(-1, "pf_flows_host: out_ptr must start at 0");
        for (int r = 0; r < nrows; ++r)
            if (out_ptr[r + 1] < out_ptr[r]) return fail(-1, "pf_flows_host: out_ptr not monotone");
        nout = out_ptr[nrows];
    }
    std::vector<void *> bufs;
    auto alloc = [&](size_t bytes, void **p) {
        cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess) bufs.push_back(*p);
        return e;
    };
    auto cleanup = [&]() {
        for (void *p : bufs) cudaFree(p);
    };
    void *dV, *dF, *dT, *dYf, *dYt, *dVn, *dSt = nullptr, *dOp = nullptr, *dOi = nullptr, *dA = nullptr, *dP = nullptr;
    const size_t vb = (size_t)nrows * n * 16, ob = (size_t)nrows * nb * 8;
    cudaError_t e;
    if ((e = alloc(vb, &dV)) != cudaSuccess || (e = alloc(nb * 4, &dF)) != cudaSuccess ||
        (e = alloc(nb * 4, &dT)) != cudaSuccess || (e = alloc(nb * 16, &dYf)) != cudaSuccess ||
        (e = alloc(nb * 16, &dYt)) != cudaSuccess || (e = alloc(nb * 8, &dVn)) != cudaSuccess ||
        (br->status && (e = alloc(nb, &dSt)) != cudaSuccess) ||
        (out_ptr && ((e = alloc((size_t)(nrows + 1) * 4, &dOp)) != cudaSuccess ||
                     (e = alloc((size_t)std::max(nout, 1) * 4, &dOi)) != cudaSuccess)) ||
        (amps && (e = alloc(ob, &dA)) != cudaSuccess) || (p_mw && (e = alloc(ob, &dP)) != cudaSuccess)) {
        cleanup();
        return cuda_fail(e, "pf_flows_host: allocation");
    }
    auto up = [&](void *d, const void *h, size_t b) { return cudaMemcpy(d, h, b, cudaMemcpyHostToDevice); };
    if ((e = up(dV, V_ri, vb)) != cudaSuccess || (e = up(dF, br->from, nb * 4)) != cudaSuccess ||
        (e = up(dT, br->to, nb * 4)) != cudaSuccess || (e = up(dYf, br->yff_ri, nb * 16)) != cudaSuccess ||
        (e = up(dYt, br->yft_ri, nb * 16)) != cudaSuccess || (e = up(dVn, br->vn_kv_from, nb * 8)) != cudaSuccess ||
        (dSt && (e = up(dSt, br->status, nb)) != cudaSuccess) ||
        (dOp && ((e = up(dOp, out_ptr, (size_t)(nrows + 1) * 4)) != cudaSuccess ||
                 (nout > 0 && (e = up(dOi, out_ids, (size_t)nout * 4)) != cudaSuccess)))) {
        cleanup();
        return cuda_fail(e, "pf_flows_host: upload");
    }
    pf_branch_set d{nb, static_cast<const int *>(dF), static_cast<const int *>(dT), static_cast<const double *>(dYf),
                    static_cast<const double *>(dYt), static_cast<const double *>(dVn),
                    static_cast<const unsigned char *>(dSt), br->sn_mva};
    int rc = pf_flows_device(&d, n, nrows, static_cast<const double *>(dV), n, nullptr, nullptr,
                             static_cast<const int *>(dOp), static_cast<const int *>(dOi), static_cast<double *>(dA),
                             static_cast<double *>(dP), nullptr);
    if (rc != 0) {
        cleanup();
        return rc;
    }
    if ((amps && (e = cudaMemcpy(amps, dA, ob, cudaMemcpyDeviceToHost)) != cudaSuccess) ||
        (p_mw && (e = cudaMemcpy(p_mw, dP, ob, cudaMemcpyDeviceToHost)) != cudaSuccess)) {
        cleanup();
        return cuda_fail(e, "pf_flows_host: download");
    }
    cleanup();
    return 0;
}


int pf_ybus_positions(const pf_plan *pl, int ncoef, const int *rows, const int *cols, int *pos) {
    if (!pl || ncoef < 0 || (ncoef > 0 && (!rows || !cols || !pos))) return fail(-1, "pf_ybus_positions: invalid argument");
    const l2g::Plan &P = pl->P;
    for (int i = 0; i < ncoef; ++i) {
        pos[i] = -1;
        const int r = rows[i], c = cols[i];
        if (r < 0 || r >= P.n || c < 0 || c >= P.n) continue;
        for (int q = P.Rp[r]; q < P.Rp[r + 1]; ++q)
            if (P.Rj[q] == c) {
                pos[i] = q;
                break;
            }
    }
    return 0;
}

static int device_sms(int *sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, dev);
    return e == cudaSuccess ? 0 : cuda_fail(e, "device query");
}

int pf_assemble_ybus_device(int nnz, const int *cptr, const int *cids, const double *r, const double *x,
                            const double *h_ri, const unsigned char *status, double *ybus_ri, void *stream) {
    if (nnz < 0 || (nnz > 0 && (!cptr || !cids || !r || !x || !h_ri || !ybus_ri)))
        return fail(-1, "pf_assemble_ybus_device: invalid argument");
    int sms = 0;
    if (device_sms(&sms) != 0) return -1;
    l2g::YbusArgs a{nnz, cptr, cids, r, x, reinterpret_cast<const double2 *>(h_ri), status,
                    reinterpret_cast<double2 *>(ybus_ri)};
    cudaError_t e = l2g::launch_assemble_ybus(a, sms, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? 0 : cuda_fail(e, "pf_assemble_ybus_device: kernel");
}

int pf_set_ybus_values_device(pf_plan *pl, const double *ybus_ri, void *stream) {
    if (!pl || !ybus_ri) return fail(-1, "pf_set_ybus_values_device: null argument");
    cudaError_t e = cudaMemcpyAsync(const_cast<double2 *>(pl->dp.Rx), ybus_ri, (size_t)pl->P.nnzY * 16,
                                    cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? 0 : cuda_fail(e, "pf_set_ybus_values_device");
}

int pf_assemble_sbus_device(const pf_sbus_layout *lay, int nsteps, const double *gen_p, const double *sgen_p,
                            const double *load_p, const double *load_q, double sn_mva, double *sbus_ri,
                            void *stream) {
    if (!lay || nsteps < 0 || lay->n <= 0 || !sbus_ri || !lay->gen_ptr || !lay->load_ptr ||
        (lay->ngen > 0 && (!lay->gen_ids || !gen_p)) || (lay->nload > 0 && (!lay->load_ids || !load_p || !load_q)) ||
        (lay->sgen_ptr && lay->nsgen > 0 && (!lay->sgen_ids || !sgen_p)))
        return fail(-1, "pf_assemble_sbus_device: invalid argument");
    int sms = 0;
    if (device_sms(&sms) != 0) return -1;
    l2g::SbusArgs a{};
    a.nsteps = nsteps;
    a.n = lay->n;
    a.ngen = lay->ngen;
    a.nsgen = lay->nsgen;
    a.nload = lay->nload;
    a.gen_ptr = lay->gen_ptr;
    a.gen_ids = lay->gen_ids;
    a.sgen_ptr = lay->sgen_ptr;
    a.sgen_ids = lay->sgen_ids;
    a.load_ptr = lay->load_ptr;
    a.load_ids = lay->load_ids;
    a.gen_p = gen_p;
    a.sgen_p = sgen_p;
    a.load_p = load_p;
    a.load_q = load_q;
    a.sn_mva = sn_mva;
    a.out = reinterpret_cast<double2 *>(sbus_ri);
    cudaError_t e = l2g::launch_assemble_sbus(a, sms, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? 0 : cuda_fail(e, "pf_assemble_sbus_device: kernel");
}

}  // extern "C"
