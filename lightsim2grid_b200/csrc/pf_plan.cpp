// Host-side symbolic analysis: Jacobian pattern, ordering, first factorisation, schedules.
#include "pf_plan.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <sstream>
#include <system_error>
#include <thread>

namespace l2g {

namespace {

// Runs f(0) ... f(n-1) on up to 8 host threads (the calls must be independent); on one thread
// when threads cannot be started.
template <typename F>
void parallel_for(int n, F f) {
    const int nt = std::min<int>(n, std::max(1, std::min(8, (int)std::thread::hardware_concurrency())));
    if (nt <= 1) {
        for (int i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<int> next(0);
    auto worker = [&]() {
        for (int i = next++; i < n; i = next++) f(i);
    };
    std::vector<std::thread> pool;
    try {
        for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    } catch (const std::system_error &) {
        // fewer threads: the calling thread and those started share the rest
    }
    worker();
    for (auto &th : pool) th.join();
}

// -------------------------------------------------------------------------------------
// Minimum-degree ordering on the symmetric pattern of A + A^T.
//
// Explicit elimination graph (Rose 1972; Tinney & Walker scheme 2): eliminating v joins
// its neighbours into a clique.  Degrees are kept in bucket lists so that the next
// minimum is found in O(1); ties go to the most recently touched node of the bucket.
// With level_slack > 0 the choice also looks at depth: every vertex carries the elimination
// level it would get (one more than the highest level of its eliminated neighbours), and among
// the vertices of degree at most the minimum + level_slack the one of lowest level is taken
// (first found on ties), which keeps the elimination tree shallow at little cost in fill.
// -------------------------------------------------------------------------------------
std::vector<int> minimum_degree(int m, const std::vector<int> &Ap, const std::vector<int> &Ai,
                                int level_slack = 0) {
    std::vector<std::vector<int>> adj(m);
    for (int j = 0; j < m; ++j)
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
            int i = Ai[p];
            if (i == j) continue;
            adj[i].push_back(j);
            adj[j].push_back(i);
        }
    for (auto &a : adj) {
        std::sort(a.begin(), a.end());
        a.erase(std::unique(a.begin(), a.end()), a.end());
    }
    // bucket lists
    std::vector<int> head(m + 1, -1), next(m, -1), prev(m, -1), deg(m);
    auto unlink = [&](int v) {
        if (prev[v] >= 0) next[prev[v]] = next[v]; else head[deg[v]] = next[v];
        if (next[v] >= 0) prev[next[v]] = prev[v];
        prev[v] = next[v] = -1;
    };
    auto link = [&](int v) {
        prev[v] = -1;
        next[v] = head[deg[v]];
        if (head[deg[v]] >= 0) prev[head[deg[v]]] = v;
        head[deg[v]] = v;
    };
    for (int v = m - 1; v >= 0; --v) {
        deg[v] = (int)adj[v].size();
        link(v);
    }
    std::vector<char> alive(m, 1);
    std::vector<int> mark(m, -1), order;
    order.reserve(m);
    int mindeg = 0, stamp = 0;
    std::vector<int> merged;
    std::vector<int> lev(m, 0);
    for (int k = 0; k < m; ++k) {
        while (mindeg <= m && head[mindeg] < 0) ++mindeg;
        int v = head[mindeg];
        if (level_slack > 0)
            for (int d = mindeg; d <= std::min(m, mindeg + level_slack); ++d)
                for (int u = head[d]; u >= 0; u = next[u])
                    if (lev[u] < lev[v]) v = u;
        unlink(v);
        alive[v] = 0;
        order.push_back(v);
        const std::vector<int> nb = adj[v];
        for (int u : nb)
            if (alive[u]) lev[u] = std::max(lev[u], lev[v] + 1);
        for (int u : nb) {
            if (!alive[u]) continue;
            merged.clear();
            ++stamp;
            mark[u] = stamp;
            mark[v] = stamp;
            for (int z : adj[u])
                if (alive[z] && mark[z] != stamp) { mark[z] = stamp; merged.push_back(z); }
            for (int z : nb)
                if (alive[z] && mark[z] != stamp) { mark[z] = stamp; merged.push_back(z); }
            adj[u].assign(merged.begin(), merged.end());
            unlink(u);
            deg[u] = (int)adj[u].size();
            link(u);
            if (deg[u] < mindeg) mindeg = deg[u];
        }
        adj[v].clear();
        adj[v].shrink_to_fit();
    }
    return order;
}

// Equivalent reordering of low elimination height (Jess & Kees 1982): the filled graph of A + A^T
// under `order` is chordal, and eliminating in rounds a maximal independent set of its
// simplicial vertices is a perfect elimination ordering of it (no fill beyond the filled
// graph's) whose rounds bound the dependency depth.  Within a round vertices keep their
// position in `order`.
std::vector<int> low_height_order(int m, const std::vector<int> &Ap, const std::vector<int> &Ai,
                                  const std::vector<int> &order) {
    std::vector<int> pos(m);
    for (int k = 0; k < m; ++k) pos[order[k]] = k;
    // symbolic elimination in `order`: the later neighbours of step k, merged into its parent's
    std::vector<std::vector<int>> up(m);
    for (int j = 0; j < m; ++j)
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
            const int a = pos[j], b = pos[Ai[p]];
            if (a == b) continue;
            up[std::min(a, b)].push_back(std::max(a, b));
        }
    std::vector<std::vector<int>> adj(m);  // filled graph, step numbering
    std::vector<int> merged;
    for (int k = 0; k < m; ++k) {
        auto &u = up[k];
        std::sort(u.begin(), u.end());
        u.erase(std::unique(u.begin(), u.end()), u.end());
        if (u.empty()) continue;
        const int par = u[0];
        for (int i : u) {
            adj[k].push_back(i);
            adj[i].push_back(k);
        }
        up[par].insert(up[par].end(), u.begin() + 1, u.end());
        std::vector<int>().swap(u);
    }
    for (auto &a : adj) std::sort(a.begin(), a.end());
    std::vector<char> alive(m, 1), simp(m, 0), taken(m, 0);
    std::vector<int> mark(m, -1), deg(m);
    int stamp = 0;
    for (int v = 0; v < m; ++v) deg[v] = (int)adj[v].size();
    auto simplicial = [&](int v) {
        ++stamp;
        for (int a : adj[v])
            if (alive[a]) mark[a] = stamp;
        for (int a : adj[v]) {
            if (!alive[a]) continue;
            int c = 0;
            for (int z : adj[a])
                if (alive[z] && mark[z] == stamp) ++c;
            if (c != deg[v] - 1) return false;
        }
        return true;
    };
    for (int v = 0; v < m; ++v) simp[v] = simplicial(v);
    std::vector<int> out;
    out.reserve(m);
    std::vector<int> round, touched;
    while ((int)out.size() < m) {
        round.clear();
        for (int v = 0; v < m; ++v) {
            if (!alive[v] || !simp[v]) continue;
            bool free = true;
            for (int a : adj[v])
                if (alive[a] && taken[a]) { free = false; break; }
            if (!free) continue;
            taken[v] = 1;
            round.push_back(v);
        }
        if (round.empty()) return order;  // not chordal: cannot happen for a filled graph
        touched.clear();
        for (int v : round) {
            alive[v] = 0;
            out.push_back(order[v]);
        }
        for (int v : round)
            for (int a : adj[v])
                if (alive[a]) {
                    --deg[a];
                    touched.push_back(a);
                }
        for (int v : round) taken[v] = 0;
        for (int a : touched) simp[a] = simplicial(a);
    }
    return out;
}

// Depth (longest dependency chain) and fill of the symbolic factorisation of A + A^T eliminated
// in `order`: the diagonal-pivot estimate of the refactorisation's levels.
int symbolic_depth(int m, const std::vector<int> &Ap, const std::vector<int> &Ai, const std::vector<int> &order,
                   long long &fill) {
    std::vector<int> pos(m);
    for (int k = 0; k < m; ++k) pos[order[k]] = k;
    std::vector<std::vector<int>> up(m);
    for (int j = 0; j < m; ++j)
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) {
            const int a = pos[j], b = pos[Ai[p]];
            if (a != b) up[std::min(a, b)].push_back(std::max(a, b));
        }
    std::vector<int> lev(m, 0);
    int depth = 0;
    fill = 0;
    for (int k = 0; k < m; ++k) {
        auto &u = up[k];
        std::sort(u.begin(), u.end());
        u.erase(std::unique(u.begin(), u.end()), u.end());
        fill += (long long)u.size();
        depth = std::max(depth, lev[k] + 1);
        for (int i : u) lev[i] = std::max(lev[i], lev[k] + 1);
        if (!u.empty()) up[u[0]].insert(up[u[0]].end(), u.begin() + 1, u.end());
        std::vector<int>().swap(u);
    }
    return depth;
}

// Minimum degree breaks ties by vertex label, and the depth of the equivalent least-depth order
// varies with those choices: orders of `trials` relabellings (the identity first, then seeded
// shuffles) are compared and the shallowest kept (then the least fill).
std::vector<int> shallow_order(int m, const std::vector<int> &Ap, const std::vector<int> &Ai, int trials,
                               int level_slack) {
    const int T = std::max(1, trials);
    // the relabellings, drawn in sequence from one seed (the identity first)
    std::vector<std::vector<int>> perm(T, std::vector<int>(m));
    unsigned seed = 0x2545f491u;
    for (int t = 0; t < T; ++t) {
        for (int i = 0; i < m; ++i) perm[t][i] = i;
        if (t > 0)
            for (int i = m - 1; i > 0; --i) {
                seed = seed * 1664525u + 1013904223u;
                std::swap(perm[t][i], perm[t][(seed >> 8) % (unsigned)(i + 1)]);
            }
    }
    std::vector<std::vector<int>> q(T);
    std::vector<int> depth(T);
    std::vector<long long> fill(T);
    parallel_for(T, [&](int t) {
        const std::vector<int> &pm = perm[t];
        std::vector<int> inv(m);
        for (int i = 0; i < m; ++i) inv[pm[i]] = i;
        // the pattern with vertex i labelled pm[i]
        std::vector<std::vector<int>> cols(m);
        for (int j = 0; j < m; ++j)
            for (int p = Ap[j]; p < Ap[j + 1]; ++p) cols[pm[j]].push_back(pm[Ai[p]]);
        std::vector<int> Bp(m + 1, 0), Bi;
        Bi.reserve(Ai.size());
        for (int j = 0; j < m; ++j) {
            std::sort(cols[j].begin(), cols[j].end());
            Bi.insert(Bi.end(), cols[j].begin(), cols[j].end());
            Bp[j + 1] = (int)Bi.size();
        }
        q[t] = low_height_order(m, Bp, Bi, minimum_degree(m, Bp, Bi, level_slack));
        for (int &v : q[t]) v = inv[v];
        depth[t] = symbolic_depth(m, Ap, Ai, q[t], fill[t]);
    });
    int best = 0;
    for (int t = 1; t < T; ++t)
        if (depth[t] < depth[best] || (depth[t] == depth[best] && fill[t] < fill[best])) best = t;
    return q[best];
}

// Builds one phase program, level after level.  All operations of a level that write the
// same value form a cluster and run on one thread, in the order they were added (so there
// are no write conflicts, no atomics and a deterministic summation order); clusters are
// spread over the threads longest-first onto the least loaded thread.  A phase is stored
// with stride `width` (threads that have work): thread t < width runs operations
// base + t, base + t + width, ...; shorter threads are padded with empty operations.  With
// `lu_base` set, the same operations are also stored in a second placement (`ops_banked`, same
// phases, widths and lengths) chosen for few shared-memory bank conflicts in the packed layout.
struct ProgramBuilder {
    Plan::Program &prog;
    int nt;
    std::vector<int> ops;          // 4 ints per operation of the current level
    std::vector<long long> key;    // written value: space (0 lu, 1 v) and index

    int lu_base = -1;              // index-space offset of the LU in the packed layout; >= 0:
                                   // order each thread's operations for few bank conflicts
    int vdummy = 0;                // index of the empty operations' scratch slot
    int lanes = 32;                // lanes served together by the shared-memory banks: a warp for
                                   // 4-byte words, a half-warp for 8-byte words (16 bank pairs)
    bool spread = false;           // clusters spread over the phase's slots (else first slots)
    // one bank placement per phase, computed by finish() on host threads
    struct BankJob {
        std::vector<int> ops, cfirst, ccount, idx;
        std::vector<std::vector<int>> per;  // the longest-first placement (the fallback)
        int width = 0, len = 0;
        size_t at = 0;  // first int of the phase in ops_banked
    };
    std::vector<BankJob> jobs;

    ProgramBuilder(Plan::Program &p, int threads) : prog(p), nt(threads) {
        prog.ops.clear();
        prog.ops_banked.clear();
        prog.base.assign(1, 0);
        prog.width.clear();
    }
    void begin() {
        ops.clear();
        key.clear();
    }
    void add(int x, int y, int z, int w, int kind) {
        ops.push_back(x);
        ops.push_back(y);
        ops.push_back(z);
        ops.push_back(w | (kind << 28));
        key.push_back(((long long)(kind == 0 ? 0 : 1) << 32) | (long long)x);
    }
    void end() {
        const int n = (int)key.size();
        if (n == 0) return;
        std::vector<int> idx(n);
        for (int i = 0; i < n; ++i) idx[i] = i;
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return key[a] < key[b]; });
        struct Cl { int first, count; };
        std::vector<Cl> cl;
        for (int i = 0; i < n;) {
            int j = i;
            while (j < n && key[idx[j]] == key[idx[i]]) ++j;
            cl.push_back({i, j - i});
            i = j;
        }
        std::stable_sort(cl.begin(), cl.end(), [](const Cl &a, const Cl &b) { return a.count > b.count; });
        const int width = std::min<int>(nt, (int)cl.size());
        std::vector<std::vector<int>> per(width);
        std::vector<std::pair<int, int>> heap;  // (load, thread), min-heap
        for (int t = 0; t < width; ++t) heap.push_back({0, t});
        auto cmp = [](const std::pair<int, int> &a, const std::pair<int, int> &b) {
            return a.first != b.first ? a.first > b.first : a.second > b.second;
        };
        std::make_heap(heap.begin(), heap.end(), cmp);
        for (const Cl &c : cl) {
            std::pop_heap(heap.begin(), heap.end(), cmp);
            auto &h = heap.back();
            for (int q = 0; q < c.count; ++q) per[h.second].push_back(idx[c.first + q]);
            h.first += c.count;
            std::push_heap(heap.begin(), heap.end(), cmp);
        }
        int len = 0;
        for (auto &v : per) len = std::max(len, (int)v.size());
        for (auto &v : per) v.resize(len, -1);
        prog.ops.resize(prog.ops.size() + 4 * (size_t)width * len);
        emit(prog.ops.data() + prog.ops.size() - 4 * (size_t)width * len, ops, per, width, len);
        if (lu_base >= 0) {
            BankJob jb;
            jb.ops = ops;
            for (const Cl &c : cl) {
                jb.cfirst.push_back(c.first);
                jb.ccount.push_back(c.count);
            }
            jb.idx = idx;
            jb.per = std::move(per);
            jb.width = width;
            jb.len = len;
            jb.at = prog.ops_banked.size();
            prog.ops_banked.resize(prog.ops_banked.size() + 4 * (size_t)width * len);
            jobs.push_back(std::move(jb));
        }
        prog.width.push_back(width);
        prog.base.push_back((int)(prog.ops.size() / 4));
    }

    // the bank placements of all phases, each into its own range of ops_banked
    void finish() {
        parallel_for((int)jobs.size(), [&](int i) {
            const BankJob &jb = jobs[i];
            const auto slot = assign_banked(jb.ops, jb.cfirst, jb.ccount, jb.idx, jb.width, jb.len);
            emit(prog.ops_banked.data() + jb.at, jb.ops, slot.empty() ? jb.per : slot, jb.width, jb.len);
        });
        jobs.clear();
    }

    // writes a phase: slot j of thread t at j * width + t (-1: empty operation)
    static void emit(int *out, const std::vector<int> &src, const std::vector<std::vector<int>> &slot, int width,
                     int len) {
        for (int j = 0; j < len; ++j)
            for (int t = 0; t < width; ++t, out += 4) {
                const int o = slot[t][j];
                if (o >= 0) std::copy(src.begin() + 4 * o, src.begin() + 4 * o + 4, out);
                else {
                    const int none[4] = {0, 0, 0, 7 << 28};
                    std::copy(none, none + 4, out);
                }
            }
    }

    // shared-memory word of field f (0 x, 1 y, 2 z, 3 w) of operation o in the packed layout
    unsigned word(const std::vector<int> &ops, int o, int f) const {
        const int kind = (unsigned)ops[4 * o + 3] >> 28;
        const int v = f == 3 ? (ops[4 * o + 3] & 0x0fffffff) : ops[4 * o + f];
        if (kind == 0) return (unsigned)(lu_base + v);
        if (kind == 2) return (unsigned)((f == 0 || f == 2) ? v : lu_base + v);
        return (unsigned)vdummy;
    }

    // Places the level's operations on (thread, slot), `len` slots per thread, so that the 32
    // operations a warp runs together touch few shared-memory words per bank (4-byte words: 32
    // banks per warp; 8-byte words: 16 bank pairs per half-warp; lanes reading one word share
    // it).  Operations writing one value (clusters of two or more) run on one thread in order,
    // placed first onto the least loaded threads as in the LPT placement: in the thread's first
    // slots, or (`spread`) each in the slot of least conflict after the previous one.  The single
    // operations then fill the free slots warp-slot by warp-slot, each lane taking the candidate
    // that adds the fewest conflicts (the written word counts twice: loaded and stored).  Greedy,
    // with the search cut where a bank's written-word conflicts alone reach the best cost found.
    std::vector<std::vector<int>> assign_banked(const std::vector<int> &ops, const std::vector<int> &cfirst,
                                                const std::vector<int> &ccount, const std::vector<int> &idx,
                                                int width, int len) const {
        const int ncl = (int)cfirst.size();
        const unsigned nb = (unsigned)lanes;  // banks (or bank pairs) per group of lanes
        std::vector<std::vector<int>> slot(width);
        std::vector<int> fill(width, 0);
        if (!spread) {
            // clusters in the first slots of the least loaded lanes, longest first
            std::vector<std::pair<int, int>> heap;
            for (int t = 0; t < width; ++t) heap.push_back({0, t});
            auto cmp = [](const std::pair<int, int> &a, const std::pair<int, int> &b) {
                return a.first != b.first ? a.first > b.first : a.second > b.second;
            };
            std::make_heap(heap.begin(), heap.end(), cmp);
            for (int c = 0; c < ncl && ccount[c] > 1; ++c) {
                std::pop_heap(heap.begin(), heap.end(), cmp);
                auto &h = heap.back();
                for (int q = 0; q < ccount[c]; ++q) slot[h.second].push_back(idx[cfirst[c] + q]);
                h.first += ccount[c];
                fill[h.second] = h.first;
                std::push_heap(heap.begin(), heap.end(), cmp);
            }
            for (auto &v : slot) v.resize(len, -1);
        } else {
            // clusters, longest first, onto a least loaded lane (as above); one lane per group
            // is tried, and the cluster's operations take, in order, the slots of least conflict
            // (cluster operations already in a warp-slot count against it, to spread them)
            for (auto &v : slot) v.assign(len, -1);
            const int ngroups = (width + lanes - 1) / lanes;
            std::vector<std::vector<unsigned>> used((size_t)ngroups * len * 4);  // distinct words
            std::vector<int> nchain((size_t)ngroups * len, 0);
            auto op_cost = [&](int o, int g, int j) {
                long long cost = 0;
                for (int f = 0; f < 4; ++f) {
                    const unsigned a = word(ops, o, f);
                    int same = 0;
                    bool present = false;
                    for (unsigned v : used[(((size_t)g * len) + j) * 4 + f]) {
                        if (v == a) { present = true; break; }
                        same += v % nb == a % nb;
                    }
                    if (!present) cost += (f == 0 ? 2 : 1) * (long long)same;
                }
                return 4 * cost + nchain[(size_t)g * len + j];
            };
            std::vector<int> pick, bpick, freeafter(len + 1);
            for (int c = 0; c < ncl && ccount[c] > 1; ++c) {
                const int k = ccount[c];
                int fmin = len;
                for (int t = 0; t < width; ++t) fmin = std::min(fmin, fill[t]);
                int bt = -1;
                long long bcost = 0;
                for (int g = 0; g < ngroups; ++g) {
                    int t = -1;
                    for (int u = g * lanes; u < std::min(width, (g + 1) * lanes); ++u)
                        if (fill[u] == fmin) { t = u; break; }
                    if (t < 0) continue;
                    // slots in order, each after the previous, leaving room for the rest
                    freeafter[len] = 0;  // free slots of this lane from j on
                    for (int j = len - 1; j >= 0; --j) freeafter[j] = freeafter[j + 1] + (slot[t][j] < 0);
                    pick.clear();
                    long long cost = 0;
                    int prev = -1;
                    for (int q = 0; q < k; ++q) {
                        int bj = -1;
                        long long bc = 0;
                        for (int j = prev + 1; j < len; ++j) {
                            if (slot[t][j] >= 0) continue;
                            if (freeafter[j + 1] < k - 1 - q) break;
                            const long long cc = op_cost(idx[cfirst[c] + q], g, j);
                            if (bj < 0 || cc < bc) { bj = j; bc = cc; }
                        }
                        if (bj < 0) return {};  // cannot happen: the lane has k free slots
                        pick.push_back(bj);
                        cost += bc;
                        prev = bj;
                    }
                    if (bt < 0 || cost < bcost) { bt = t; bcost = cost; bpick = pick; }
                }
                if (bt < 0) return {};
                const int g = bt / lanes;
                for (int q = 0; q < k; ++q) {
                    const int o = idx[cfirst[c] + q], j = bpick[q];
                    slot[bt][j] = o;
                    ++nchain[(size_t)g * len + j];
                    for (int f = 0; f < 4; ++f) {
                        const unsigned a = word(ops, o, f);
                        auto &l = used[(((size_t)g * len) + j) * 4 + f];
                        if (std::find(l.begin(), l.end(), a) == l.end()) l.push_back(a);
                    }
                }
                fill[bt] += k;
            }
        }
        // single operations, bucketed by the bank of the word they write
        std::vector<std::vector<int>> bucket(nb);
        for (int c = 0; c < ncl; ++c)
            if (ccount[c] == 1) bucket[word(ops, idx[cfirst[c]], 0) % nb].push_back(idx[cfirst[c]]);
        for (auto &b : bucket) std::reverse(b.begin(), b.end());  // pop from the back in order
        int left = 0;
        for (auto &b : bucket) left += (int)b.size();
        for (int j = 0; j < len && left > 0; ++j)
            for (int q0 = 0; q0 < width && left > 0; q0 += lanes) {
                const int q1 = std::min(width, q0 + lanes);
                std::vector<std::vector<unsigned>> seen[4];
                for (auto &sf : seen) sf.assign(nb, {});
                auto add = [&](int o) {
                    for (int f = 0; f < 4; ++f) {
                        const unsigned a = word(ops, o, f);
                        auto &s2 = seen[f][a % nb];
                        if (std::find(s2.begin(), s2.end(), a) == s2.end()) s2.push_back(a);
                    }
                };
                for (int t = q0; t < q1; ++t)
                    if (slot[t][j] >= 0) add(slot[t][j]);
                for (int t = q0; t < q1 && left > 0; ++t) {
                    if (slot[t][j] >= 0) continue;
                    int bb = -1, bi = -1;
                    long long bc = 0;
                    for (int bk = 0; bk < (int)nb && !(bb >= 0 && bc == 0); ++bk) {
                        auto &b = bucket[bk];
                        if (!seen[0][bk].empty() && bb >= 0 && bc <= 2 * (long long)seen[0][bk].size()) continue;
                        for (int u = 0; u < (int)b.size(); ++u) {
                            const int o = b[b.size() - 1 - u];
                            long long cost = 0;
                            for (int f = 0; f < 4; ++f) {
                                const unsigned a = word(ops, o, f);
                                const auto &s2 = seen[f][a % nb];
                                if (std::find(s2.begin(), s2.end(), a) == s2.end()) cost += (f == 0 ? 2 : 1) * (long long)s2.size();
                            }
                            if (bb < 0 || cost < bc) { bb = bk; bi = u; bc = cost; }
                            if (bc == 0) break;
                        }
                    }
                    auto &b = bucket[bb];
                    const size_t at = b.size() - 1 - bi;
                    const int o = b[at];
                    b.erase(b.begin() + at);
                    --left;
                    slot[t][j] = o;
                    add(o);
                }
            }
        if (left > 0) return {};  // cannot happen: the free slots hold every single operation
        return slot;
    }
};

}  // namespace

int compact_lu_offset(int m) { return (m + 1 + 3) & ~3; }

bool compact_fits(const Plan &P) { return (long long)compact_lu_offset(P.m) + P.nnzLU <= 65536; }

void compact_ops(const Plan::Program &pr, int m, std::vector<unsigned> &out, int lu_offset) {
    const unsigned L = (unsigned)(lu_offset >= 0 ? lu_offset : compact_lu_offset(m)), dummy = (unsigned)m;
    // the bank-conflict placement assumes the default layout
    const std::vector<int> &ops = lu_offset < 0 && !pr.ops_banked.empty() ? pr.ops_banked : pr.ops;
    const int n = pr.nops();
    out.resize(2 * (size_t)n);
    for (int o = 0; o < n; ++o) {
        const unsigned x = (unsigned)ops[4 * o], y = (unsigned)ops[4 * o + 1], z = (unsigned)ops[4 * o + 2];
        const unsigned w = (unsigned)ops[4 * o + 3] & 0x0fffffffu, kind = (unsigned)ops[4 * o + 3] >> 28;
        unsigned X = dummy, Y = dummy, Z = dummy, W = dummy;
        if (kind == 0u) {
            X = L + x; Y = L + y; Z = L + z; W = L + w;
        } else if (kind == 2u) {
            X = x; Y = L + y; Z = z; W = L + w;
        }
        out[2 * (size_t)o] = X | (Y << 16);
        out[2 * (size_t)o + 1] = Z | (W << 16);
    }
}

long long smem_wavefronts(const Plan &P, const Plan::Program &pr) {
    const int G = P.bank_lanes;
    if (G <= 0) return 0;
    std::vector<unsigned> c;
    compact_ops(pr, P.m, c, -1);
    long long total = 0;
    std::vector<unsigned> u;
    for (int p = 0; p < pr.nphases(); ++p) {
        const int b0 = pr.base[p], w = pr.width[p], len = (pr.base[p + 1] - b0) / w;
        for (int j = 0; j < len; ++j)
            for (int q = 0; q < w; q += G)
                for (int f = 0; f < 4; ++f) {
                    u.clear();
                    for (int t = q; t < std::min(w, q + G); ++t) {
                        const size_t o = (size_t)b0 + t + (size_t)j * w;
                        const unsigned v = (f & 1) ? c[2 * o + (f >> 1)] >> 16 : c[2 * o + (f >> 1)] & 0xffffu;
                        u.push_back(v);
                    }
                    std::sort(u.begin(), u.end());
                    u.erase(std::unique(u.begin(), u.end()), u.end());
                    int cnt[32] = {0}, mx = 0;
                    for (unsigned v : u) mx = std::max(mx, ++cnt[v % G]);
                    total += (f == 0 ? 2 : 1) * (long long)mx;
                }
    }
    return total;
}

void build_tile_program(const Plan::Program &pr, int nwarps, int chunk, TileProgram &out) {
    out.ops.clear();
    out.phase.clear();
    int nchunks = 0;
    std::vector<int> idx;
    std::vector<long long> key;
    for (int p = 0; p < pr.nphases(); ++p) {
        // the phase's operations in program order (slot after slot), padding dropped
        idx.clear();
        key.clear();
        for (int k = pr.base[p]; k < pr.base[p + 1]; ++k) {
            const unsigned kind = (unsigned)pr.ops[4 * (size_t)k + 3] >> 28;
            if (kind == 7u) continue;
            idx.push_back(k);
            key.push_back(((long long)(kind == 0u ? 0 : 1) << 32) | (long long)pr.ops[4 * (size_t)k]);
        }
        const int n = (int)idx.size();
        std::vector<int> ord(n);
        for (int i = 0; i < n; ++i) ord[i] = i;
        // a written value's operations sit on one slot in program order; the stable sort keeps
        // that order inside each group
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return key[a] < key[b]; });
        struct Group { int first, count; };
        std::vector<Group> groups;
        for (int i = 0; i < n;) {
            int j = i;
            while (j < n && key[ord[j]] == key[ord[i]]) ++j;
            groups.push_back({i, j - i});
            i = j;
        }
        // operand locality: groups ordered by the pivot and the U entry of their first operation
        // (consecutive groups then share the pivot, the U entry or the pivot's L column), and cut
        // into nwarps contiguous runs of about equal operation counts
        auto okey = [&](const Group &g) {
            const int *o = &pr.ops[4 * (size_t)idx[ord[g.first]]];
            return std::make_pair((long long)(o[3] & 0x0fffffff), ((long long)o[2] << 32) | (unsigned)o[1]);
        };
        std::stable_sort(groups.begin(), groups.end(), [&](const Group &a, const Group &b) { return okey(a) < okey(b); });
        std::vector<std::vector<int>> per(nwarps);
        {
            long long done = 0;
            int w = 0;
            for (const Group &g : groups) {
                // move to the next warp once this one holds its share of the phase's operations
                while (w < nwarps - 1 && done >= (long long)n * (w + 1) / nwarps) ++w;
                for (int q = 0; q < g.count; ++q) per[w].push_back(idx[ord[g.first + q]]);
                done += g.count;
            }
        }
        int rounds = 0;
        for (auto &v : per) rounds = std::max(rounds, (int)((v.size() + chunk - 1) / chunk));
        out.phase.push_back(nchunks);
        out.phase.push_back(rounds);
        for (int r = 0; r < rounds; ++r)
            for (int w = 0; w < nwarps; ++w)
                for (int c = 0; c < chunk; ++c) {
                    const size_t q = (size_t)r * chunk + c;
                    if (q < per[w].size()) {
                        const int k = per[w][q];
                        out.ops.insert(out.ops.end(), pr.ops.begin() + 4 * (size_t)k,
                                       pr.ops.begin() + 4 * (size_t)k + 4);
                    } else {
                        const int none[4] = {0, 0, 0, 7 << 28};
                        out.ops.insert(out.ops.end(), none, none + 4);
                    }
                }
        nchunks += rounds * nwarps;
    }
}

void fdpf_lu_offsets(const Plan &P, int &off0, int &off1, bool &fits) {
    const int x = std::max(compact_lu_offset(P.sub[0].m), compact_lu_offset(P.sub[1].m));
    off0 = x;
    off1 = x + ((P.sub[0].nnzLU + 3) & ~3);
    fits = (long long)off1 + P.sub[1].nnzLU <= 65536;
}

void host_jacobian(const Plan &P, const cplx *Yx, const cplx *V, std::vector<double> &Jx) {
    const int n = P.n;
    std::vector<cplx> Ibus(n, 0.0), dVm(P.nnzY), dVa(P.nnzY);
    for (int c = 0; c < n; ++c)
        for (int p = P.Yp[c]; p < P.Yp[c + 1]; ++p) Ibus[P.Yi[p]] += Yx[p] * V[c];
    const cplx jj(0.0, 1.0);
    for (int c = 0; c < n; ++c) {
        cplx vn_c = V[c] / std::abs(V[c]);
        for (int p = P.Yp[c]; p < P.Yp[c + 1]; ++p) {
            int r = P.Yi[p];
            cplx a = std::conj(Yx[p] * vn_c) * V[r];
            cplx b = Yx[p] * V[c];
            if (r == c) {
                a += std::conj(Ibus[r]) * (V[r] / std::abs(V[r]));
                b -= Ibus[r];
            }
            dVm[p] = a;
            dVa[p] = std::conj(-b) * (jj * V[r]);
        }
    }
    Jx.assign(P.Ji.size(), 0.0);
    for (size_t t = 0; t < P.Ji.size(); ++t) {
        int s = P.jsrc[t];
        if (s < 0) { Jx[t] = P.jconst[t]; continue; }
        switch (P.jkind[t]) {
            case 0: Jx[t] = dVa[s].real(); break;
            case 1: Jx[t] = dVa[s].imag(); break;
            case 2: Jx[t] = dVm[s].real(); break;
            default: Jx[t] = dVm[s].imag(); break;
        }
    }
}

// Ybus in canonical CSC form: valid pointers, sorted rows without duplicates.
int check_ybus(int n, const int *Yp, const int *Yi, std::string &msg) {
    if (Yp[0] != 0 || Yp[n] < n) {
        msg = "build_plan: Ybus column pointer is invalid";
        return NotInitError;
    }
    for (int c = 0; c < n; ++c) {
        if (Yp[c + 1] < Yp[c]) { msg = "build_plan: Ybus column pointer is not monotone"; return NotInitError; }
        for (int p = Yp[c]; p < Yp[c + 1]; ++p) {
            if (Yi[p] < 0 || Yi[p] >= n) { msg = "build_plan: Ybus row index out of range"; return NotInitError; }
            if (p > Yp[c] && Yi[p] <= Yi[p - 1]) {
                msg = "build_plan: Ybus is not in canonical CSC form (sorted, no duplicates)";
                return NotInitError;
            }
        }
    }
    return NoError;
}

// CSR copy of P's Ybus (pattern, values, CSC -> CSR position map).
void make_csr(Plan &P) {
    const int n = P.n;
    P.Rp.assign(n + 1, 0);
    for (int p = 0; p < P.nnzY; ++p) P.Rp[P.Yi[p] + 1]++;
    for (int r = 0; r < n; ++r) P.Rp[r + 1] += P.Rp[r];
    P.Rj.assign(P.nnzY, 0);
    P.Rrow.assign(P.nnzY, 0);
    P.csr_of_csc.assign(P.nnzY, 0);
    P.Rx.assign(P.nnzY, 0.0);
    std::vector<int> fp(P.Rp.begin(), P.Rp.end() - 1);
    for (int c = 0; c < n; ++c)
        for (int p = P.Yp[c]; p < P.Yp[c + 1]; ++p) {
            int r = P.Yi[p];
            int d = fp[r]++;
            P.Rj[d] = c;
            P.Rrow[d] = r;
            P.csr_of_csc[p] = d;
            P.Rx[d] = P.Yx[p];
        }
}

// Ordering, first factorisation with threshold partial pivoting, LU layout, phase programs and
// fill maps for the matrix whose pattern is P.Jp / P.Ji (m = P.m columns), whose entry t takes
// its values from Ybus position jsrc[t] (part jkind[t]) or the constant jconst[t] (jsrc < 0),
// and whose values for the first factorisation are Jx.
// Dense tail of a plan.  The fill of a grid with long-range branches gathers in the last
// columns of the elimination order (minimum degree leaves the dense separator for last), where
// the phase programs would run hundreds of levels of scattered single updates.  When the
// trailing block of the largest size tail_k in [kTailMin, kTailMax] whose LU pattern is at least
// kTailDensity full exists, steps [tail_ct, m) become a dense tail: the factor program keeps the
// updates by the pivots before tail_ct (the Schur complement the sparse part contributes to the
// block) and their pushes, the forward program the pushes of those pivots, and the backward
// program the pushes into the rows before tail_ct (those of the block's columns first, at level
// 0).  The kernel gathers the block into a dense matrix after the factor program, factorises it
// without pivoting (the plan's pivots are already in the block's order) and runs the block's
// substitutions densely, in the programs' conventions (undivided backward values).
void choose_tail(Plan &P) {
    const int m = P.m;
    P.tail_ct = m;
    P.tail_k = 0;
    P.tail_map.clear();
    if (m < kTailMin) return;
    // entries of the trailing block from step c on: LU positions with min(row, column) >= c
    std::vector<long long> cnt(m + 1, 0);
    for (int k = 0; k < m; ++k)
        for (int p = P.colstart[k]; p < P.colstart[k + 1]; ++p) cnt[std::min(P.Urow_k[p], k)]++;
    for (int c = m - 1; c >= 0; --c) cnt[c] += cnt[c + 1];
    int best = 0;
    for (int k = kTailMin; k <= std::min(kTailMax, m); ++k)
        if ((double)cnt[m - k] >= kTailDensity * (double)k * (double)k) best = k;
    if (best == 0) return;
    const int ct = m - best;
    P.tail_ct = ct;
    P.tail_k = best;
    P.tail_map.assign((size_t)best * best, -1);
    for (int k = ct; k < m; ++k)
        for (int p = P.colstart[k]; p < P.colstart[k + 1]; ++p) {
            const int r = P.Urow_k[p];
            if (r >= ct) P.tail_map[(size_t)(r - ct) * best + (k - ct)] = p;
        }
}

int analyze_lu(Plan &P, const std::vector<double> &Jx, const PlanOptions &opt, std::string &msg) {
    const int m = P.m;
    std::ostringstream err;
    // ---------------------------------------------------------------- ordering
    P.q = opt.order_trials > 0 ? shallow_order(m, P.Jp, P.Ji, opt.order_trials, opt.level_slack)
                               : minimum_degree(m, P.Jp, P.Ji, opt.level_slack);
    P.qinv.assign(m, 0);
    for (int k = 0; k < m; ++k) P.qinv[P.q[k]] = k;

    // ---------------------------------------------------------------- first factorisation
    P.pinv.assign(m, -1);
    P.prow.assign(m, -1);
    std::vector<std::vector<int>> Lrows(m), Ucols(m);  // Lrows: J rows (later steps), Ucols: steps
    std::vector<std::vector<double>> Lval(m);
    {
        std::vector<double> x(m, 0.0);
        std::vector<int> visited(m, -1), stack, topo, headp(m);
        stack.reserve(m);
        topo.reserve(m);
        for (int k = 0; k < m; ++k) {
            const int j = P.q[k];
            topo.clear();
            // depth-first reach through the columns of L already computed
            for (int p = P.Jp[j]; p < P.Jp[j + 1]; ++p) {
                int r0 = P.Ji[p];
                if (visited[r0] == k) continue;
                stack.clear();
                stack.push_back(r0);
                visited[r0] = k;
                headp[r0] = 0;
                while (!stack.empty()) {
                    int r = stack.back();
                    int c = P.pinv[r];
                    bool pushed = false;
                    if (c >= 0) {
                        const std::vector<int> &lr = Lrows[c];
                        while (headp[r] < (int)lr.size()) {
                            int r2 = lr[headp[r]++];
                            if (visited[r2] == k) continue;
                            visited[r2] = k;
                            headp[r2] = 0;
                            stack.push_back(r2);
                            pushed = true;
                            break;
                        }
                    }
                    if (!pushed) {
                        stack.pop_back();
                        topo.push_back(r);
                    }
                }
            }
            std::reverse(topo.begin(), topo.end());
            for (int r : topo) x[r] = 0.0;
            for (int p = P.Jp[j]; p < P.Jp[j + 1]; ++p) x[P.Ji[p]] = Jx[p];
            for (int r : topo) {
                int c = P.pinv[r];
                if (c < 0) continue;
                double xr = x[r];
                const std::vector<int> &lr = Lrows[c];
                const std::vector<double> &lv = Lval[c];
                for (size_t s = 0; s < lr.size(); ++s) x[lr[s]] -= lv[s] * xr;
            }
            int piv = -1;
            double amax = -1.0;
            for (int r : topo) {
                if (P.pinv[r] >= 0) continue;
                double a = std::fabs(x[r]);
                if (a > amax) { amax = a; piv = r; }
            }
            if (piv < 0 || !(amax > 0.0) || !std::isfinite(amax)) {
                err << "build_plan: the first matrix is singular (step " << k << ")";
                msg = err.str();
                return SolverFactor;
            }
            if (visited[j] == k && P.pinv[j] < 0 && std::fabs(x[j]) >= opt.pivot_threshold * amax) piv = j;
            const double pivot = x[piv];
            P.pinv[piv] = k;
            P.prow[k] = piv;
            for (int r : topo) {
                if (r == piv) continue;
                int c = P.pinv[r];
                if (c >= 0) Ucols[k].push_back(c);
                else {
                    Lrows[k].push_back(r);
                    Lval[k].push_back(x[r] / pivot);
                }
            }
        }
    }
    // rows of L to step numbering, sorted
    for (int k = 0; k < m; ++k) {
        for (int &r : Lrows[k]) r = P.pinv[r];
        std::sort(Lrows[k].begin(), Lrows[k].end());
        std::sort(Ucols[k].begin(), Ucols[k].end());
        Lval[k].clear();
        Lval[k].shrink_to_fit();
    }

    // ---------------------------------------------------------------- LU layout
    P.colstart.assign(m + 1, 0);
    P.dpos.assign(m, 0);
    P.lstart.assign(m, 0);
    P.lcount.assign(m, 0);
    int pos = 0;
    for (int k = 0; k < m; ++k) {
        P.colstart[k] = pos;
        pos += (int)Ucols[k].size();
        P.dpos[k] = pos++;
        P.lstart[k] = pos;
        P.lcount[k] = (int)Lrows[k].size();
        pos += P.lcount[k];
    }
    P.colstart[m] = pos;
    P.nnzLU = pos;
    P.Urow_k.assign(pos, 0);
    for (int k = 0; k < m; ++k) {
        for (size_t t = 0; t < Ucols[k].size(); ++t) P.Urow_k[P.colstart[k] + t] = Ucols[k][t];
        P.Urow_k[P.dpos[k]] = k;
        for (int t = 0; t < P.lcount[k]; ++t) P.Urow_k[P.lstart[k] + t] = Lrows[k][t];
    }

    // ---------------------------------------------------------------- phase programs
    if (P.nnzLU >= (1 << 28) || m >= (1 << 28)) {
        msg = "build_plan: LU too large for the operation encoding";
        return SolverAnalyze;
    }
    // the bank placement serves the packed layout: only where its 16-bit indices fit and the
    // LU, at the plan's element size, can fit the 227 KB of shared memory of a CTA
    const int packed_lu_base = compact_fits(P) && (size_t)(compact_lu_offset(m) + P.nnzLU) * opt.elem_bytes <= 232448
                                   ? compact_lu_offset(m)
                                   : -1;
    P.bank_lanes = packed_lu_base >= 0 ? (opt.elem_bytes == 8 ? 16 : 32) : 0;
    // a dense tail only where the LU cannot sit in shared memory (no packed layout)
    P.tail_ct = m;
    P.tail_k = 0;
    P.tail_map.clear();
    if (opt.dense_tail && packed_lu_base < 0) choose_tail(P);
    const int ct = P.tail_ct;
    // U row lists: for pivot c, the columns j > c with U(c, j) != 0 and the position of U(c, j)
    std::vector<std::vector<std::pair<int, int>>> urows(m);
    for (int k = 0; k < m; ++k)
        for (size_t t = 0; t < Ucols[k].size(); ++t) urows[Ucols[k][t]].push_back({k, P.colstart[k] + (int)t});
    // L row lists: for row i, the columns k < i with L(i, k) != 0
    std::vector<std::vector<int>> lrows(m);
    for (int k = 0; k < m; ++k)
        for (int i : Lrows[k]) lrows[i].push_back(k);

    // refactorisation levels: a pivot is applied once every pivot updating its column is done
    std::vector<int> level(m, 0);
    P.flops_refactor = 0;
    int nlev = 0;
    for (int k = 0; k < m; ++k) {
        int lv = 0;
        for (int c : Ucols[k]) lv = std::max(lv, level[c] + 1);
        level[k] = lv;
        nlev = std::max(nlev, lv + 1);
        for (int c : Ucols[k]) P.flops_refactor += P.lcount[c];
    }
    P.colleve = level;
    P.levels_refactor = nlev;
    // level of the fused forward push of pivot k: its L column final (level[k]) and y(k)
    // final (every push into it done).  L columns are kept undivided; consumers divide by
    // the pivot.
    std::vector<int> plev(m, 0);
    int nplev = nlev;
    for (int k = 0; k < m; ++k) {
        int lv = level[k];
        for (int kp : lrows[k]) lv = std::max(lv, plev[kp] + 1);
        plev[k] = lv;
        nplev = std::max(nplev, lv + 1);
    }
    std::vector<std::vector<int>> bylevel(nlev), bypush(nplev);
    for (int k = 0; k < m; ++k) {
        bylevel[level[k]].push_back(k);
        if (opt.fuse_forward) bypush[plev[k]].push_back(k);
    }
    std::vector<int> rowpos(m, -1);
    {
        ProgramBuilder B(P.factor, opt.threads);
        B.lu_base = packed_lu_base;
        B.vdummy = m;
        B.lanes = opt.elem_bytes == 8 ? 16 : 32;
        B.spread = opt.spread_clusters;
        for (int l = 0; l < nplev; ++l) {
            B.begin();
            if (l < nlev)
                for (int c : bylevel[l]) {
                    if (c >= ct) continue;  // the dense tail factorises the block
                    for (auto &e : urows[c]) {
                        const int j = e.first;
                        for (int p = P.colstart[j]; p < P.colstart[j + 1]; ++p) rowpos[P.Urow_k[p]] = p;
                        for (int t = 0; t < P.lcount[c]; ++t) {
                            int d = rowpos[Lrows[c][t]];
                            if (d < 0) {
                                msg = "build_plan: internal error, LU pattern is not closed";
                                return SolverAnalyze;
                            }
                            B.add(d, P.lstart[c] + t, e.second, P.dpos[c], 0);
                        }
                        for (int p = P.colstart[j]; p < P.colstart[j + 1]; ++p) rowpos[P.Urow_k[p]] = -1;
                    }
                }
            for (int k : bypush[l]) {
                if (k >= ct) continue;
                for (int t = 0; t < P.lcount[k]; ++t) B.add(Lrows[k][t], P.lstart[k] + t, k, P.dpos[k], 2);
            }
            B.end();
        }
        B.finish();
    }
    {
        // backward substitution U z = y, from the last pivot: blevel(k) = 1 + max over U(k, j)
        std::vector<int> blev(m, 0);
        int nb = 0;
        // (with a dense tail, the block's values are final before the program: its columns push
        // into the rows before the block at level 0)
        for (int k = m - 1; k >= 0; --k) {
            int lv = 0;
            if (k < ct)
                for (auto &e : urows[k]) lv = std::max(lv, blev[e.first] + 1);
            blev[k] = lv;
            nb = std::max(nb, lv + 1);
        }
        std::vector<std::vector<int>> byb(nb);
        for (int k = 0; k < m; ++k) byb[blev[k]].push_back(k);
        P.levels_bwd = nb;
        // z(k) is kept undivided by U(k, k): a push divides by the pivot, and one scaling pass
        // after the program divides every z(k) (no per-pivot division operations)
        ProgramBuilder B(P.backward, opt.threads);
        B.lu_base = packed_lu_base;
        B.vdummy = m;
        B.lanes = opt.elem_bytes == 8 ? 16 : 32;
        B.spread = opt.spread_clusters;
        for (int l = 0; l < nb; ++l) {
            B.begin();
            for (int k : byb[l])
                for (int p = P.colstart[k]; p < P.dpos[k]; ++p)
                    if (P.Urow_k[p] < ct) B.add(P.Urow_k[p], p, k, P.dpos[k], 2);
            B.end();
        }
        B.finish();
    }
    {
        // forward substitution L y = b on its own: flevel(k) = 1 + max over L(k, k')
        std::vector<int> flev(m, 0);
        int nf = 0;
        for (int k = 0; k < m; ++k) {
            int lv = 0;
            for (int kp : lrows[k]) lv = std::max(lv, flev[kp] + 1);
            flev[k] = lv;
            nf = std::max(nf, lv + 1);
        }
        std::vector<std::vector<int>> byf(nf);
        for (int k = 0; k < m; ++k) byf[flev[k]].push_back(k);
        P.levels_fwd = nf;
        ProgramBuilder B(P.forward, opt.threads);
        B.lu_base = packed_lu_base;
        B.vdummy = m;
        B.lanes = opt.elem_bytes == 8 ? 16 : 32;
        B.spread = opt.spread_clusters;
        for (int l = 0; l < nf; ++l) {
            B.begin();
            for (int k : byf[l]) {
                if (k >= ct) continue;
                for (int t = 0; t < P.lcount[k]; ++t) B.add(Lrows[k][t], P.lstart[k] + t, k, P.dpos[k], 2);
            }
            B.end();
        }
        B.finish();
    }

    // ---------------------------------------------------------------- J fill maps
    P.ytarget.assign(4 * (size_t)P.nnzY, -1);
    P.yjpos.assign(4 * (size_t)P.nnzY, -1);
    std::vector<char> covered(P.nnzLU, 0);
    for (int jc = 0; jc < m; ++jc) {
        int k = P.qinv[jc];
        for (int p = P.colstart[k]; p < P.colstart[k + 1]; ++p) rowpos[P.Urow_k[p]] = p;
        for (int t = P.Jp[jc]; t < P.Jp[jc + 1]; ++t) {
            int lu = rowpos[P.pinv[P.Ji[t]]];
            if (lu < 0) { msg = "build_plan: internal error, J entry outside the LU pattern"; return SolverAnalyze; }
            covered[lu] = 1;
            if (P.jsrc[t] < 0) {
                P.cpos.push_back(lu);
                P.cval.push_back(P.jconst[t]);
                P.cjpos.push_back(t);
            } else {
                int d = P.csr_of_csc[P.jsrc[t]];
                P.ytarget[4 * (size_t)d + P.jkind[t]] = lu;
                P.yjpos[4 * (size_t)d + P.jkind[t]] = t;
            }
        }
        for (int p = P.colstart[k]; p < P.colstart[k + 1]; ++p) rowpos[P.Urow_k[p]] = -1;
    }
    for (int p = 0; p < P.nnzLU; ++p)
        if (!covered[p]) P.fillpos.push_back(p);

    return NoError;
}

int build_plan(Plan &P, int n, const int *Yp, const int *Yi, const cplx *Yx, const cplx *V0, const cplx *Sbus,
               const int *slack_ids, int nslack, const double *weights, const int *pv, int npv_in, const int *pq,
               int npq, bool distributed, const PlanOptions &opt, std::string &msg) {
    (void)Sbus;
    P = Plan();
    std::ostringstream err;
    if (n <= 0 || nslack <= 0) {
        msg = "build_plan: the grid needs at least one bus and one slack bus";
        return NotInitError;
    }
    if (check_ybus(n, Yp, Yi, msg) != NoError) return NotInitError;
    std::vector<int> role(n, 0);  // 0 none, 1 slack, 2 pv, 3 pq
    for (int t = 0; t < nslack; ++t) {
        if (slack_ids[t] < 0 || slack_ids[t] >= n) { msg = "build_plan: slack id out of range"; return NotInitError; }
        role[slack_ids[t]] = 1;
    }
    for (int t = 0; t < npv_in; ++t) {
        if (pv[t] < 0 || pv[t] >= n || role[pv[t]] != 0) {
            msg = "build_plan: a PV bus is out of range, repeated or also a slack";
            return NotInitError;
        }
        role[pv[t]] = 2;
    }
    for (int t = 0; t < npq; ++t) {
        if (pq[t] < 0 || pq[t] >= n || role[pq[t]] != 0) {
            msg = "build_plan: a PQ bus is out of range, repeated or also PV / slack";
            return NotInitError;
        }
        role[pq[t]] = 3;
    }
    P.n = n;
    P.nnzY = Yp[n];
    P.Yp.assign(Yp, Yp + n + 1);
    P.Yi.assign(Yi, Yi + P.nnzY);
    P.Yx.assign(Yx, Yx + P.nnzY);
    P.distributed = distributed;
    P.slack0 = slack_ids[0];
    P.slack_ids.assign(slack_ids, slack_ids + nslack);
    P.weights.assign(weights, weights + n);
    // retrieve_pv_with_slack (src/powerflow_algorithm/BaseAlgo.hpp:201-216)
    if (distributed)
        for (int t = 1; t < nslack; ++t) P.mypv.push_back(slack_ids[t]);
    P.mypv.insert(P.mypv.end(), pv, pv + npv_in);
    P.pq.assign(pq, pq + npq);
    P.npv = (int)P.mypv.size();
    P.npq = npq;
    P.pvpq = P.mypv;
    P.pvpq.insert(P.pvpq.end(), pq, pq + npq);
    P.npvpq = P.npv + npq;
    P.off = distributed ? 1 : 0;
    P.m = P.npvpq + npq + P.off;
    const int m = P.m;
    if (m == 0) { msg = "build_plan: no PV or PQ bus"; return NotInitError; }

    make_csr(P);

    // ---------------------------------------------------------------- Jacobian pattern
    std::vector<int> pvpq_inv(n, -1), pq_inv(n, -1);
    for (int t = 0; t < P.npvpq; ++t) pvpq_inv[P.pvpq[t]] = t;
    for (int t = 0; t < npq; ++t) pq_inv[P.pq[t]] = t;
    const int off = P.off, npvpq = P.npvpq;
    struct Trip { int row, col, src; uint8_t kind; double val; };
    std::vector<Trip> T;
    T.reserve(4 * (size_t)P.nnzY + n + 4);
    for (int c = 0; c < npvpq; ++c) {
        int bus = P.pvpq[c];
        for (int p = Yp[bus]; p < Yp[bus + 1]; ++p)
            if (pvpq_inv[Yi[p]] >= 0) T.push_back({pvpq_inv[Yi[p]] + off, c + off, p, 0, 0.0});
        for (int p = Yp[bus]; p < Yp[bus + 1]; ++p)
            if (pq_inv[Yi[p]] >= 0) T.push_back({npvpq + pq_inv[Yi[p]] + off, c + off, p, 1, 0.0});
    }
    for (int c = 0; c < npq; ++c) {
        int bus = P.pq[c];
        for (int p = Yp[bus]; p < Yp[bus + 1]; ++p)
            if (pvpq_inv[Yi[p]] >= 0) T.push_back({pvpq_inv[Yi[p]] + off, npvpq + c + off, p, 2, 0.0});
        for (int p = Yp[bus]; p < Yp[bus + 1]; ++p)
            if (pq_inv[Yi[p]] >= 0) T.push_back({npvpq + pq_inv[Yi[p]] + off, npvpq + c + off, p, 3, 0.0});
    }
    if (distributed) {
        const int s0 = P.slack0;
        for (int c = 0; c < n; ++c) {
            if (pvpq_inv[c] < 0) continue;
            for (int p = Yp[c]; p < Yp[c + 1]; ++p)
                if (Yi[p] == s0) T.push_back({0, pvpq_inv[c] + 1, p, 0, 0.0});
        }
        for (int c = 0; c < n; ++c) {
            if (pq_inv[c] < 0) continue;
            for (int p = Yp[c]; p < Yp[c + 1]; ++p)
                if (Yi[p] == s0) T.push_back({0, npvpq + pq_inv[c] + 1, p, 2, 0.0});
        }
        T.push_back({0, 0, -1, 0, weights[s0]});
        for (int t = 0; t < npvpq; ++t) {
            double sw = weights[P.pvpq[t]];
            if (std::fabs(sw) > 1e-7) T.push_back({t + 1, 0, -1, 0, sw});
        }
    }
    std::stable_sort(T.begin(), T.end(), [](const Trip &a, const Trip &b) {
        return a.col != b.col ? a.col < b.col : a.row < b.row;
    });
    const int nnzJ = (int)T.size();
    P.Jp.assign(m + 1, 0);
    P.Ji.resize(nnzJ);
    P.jsrc.resize(nnzJ);
    P.jkind.resize(nnzJ);
    P.jconst.assign(nnzJ, 0.0);
    for (int t = 0; t < nnzJ; ++t) {
        if (t > 0 && T[t].col == T[t - 1].col && T[t].row == T[t - 1].row) {
            msg = "build_plan: duplicate Jacobian entry (is a bus both slack and PV/PQ?)";
            return NotInitError;
        }
        P.Jp[T[t].col + 1]++;
        P.Ji[t] = T[t].row;
        P.jsrc[t] = T[t].src;
        P.jkind[t] = T[t].kind;
        P.jconst[t] = T[t].val;
    }
    for (int c = 0; c < m; ++c) P.Jp[c + 1] += P.Jp[c];

    // ---------------------------------------------------------------- LU analysis
    {
        std::vector<cplx> Vinit(V0, V0 + n);
        std::vector<double> Jx;
        host_jacobian(P, P.Yx.data(), Vinit.data(), Jx);
        const int rc = analyze_lu(P, Jx, opt, msg);
        if (rc != NoError) return rc;
    }

    // ---------------------------------------------------------------- bus maps
    P.xP.assign(n, -1);
    P.xQ.assign(n, -1);
    P.xVa.assign(n, -1);
    P.xVm.assign(n, -1);
    for (int b = 0; b < n; ++b) {
        int fP = -1, fQ = -1;
        if (distributed && b == P.slack0) fP = 0;
        else if (pvpq_inv[b] >= 0) fP = pvpq_inv[b] + off;
        if (pq_inv[b] >= 0) fQ = npvpq + pq_inv[b] + off;
        if (fP >= 0) P.xP[b] = P.pinv[fP];
        if (fQ >= 0) P.xQ[b] = P.pinv[fQ];
        if (pvpq_inv[b] >= 0) P.xVa[b] = P.qinv[pvpq_inv[b] + off];
        if (pq_inv[b] >= 0) P.xVm[b] = P.qinv[npvpq + pq_inv[b] + off];
    }
    if (distributed) P.xSlack = P.qinv[0];
    return NoError;
}

int build_dc_plan(Plan &P, int n, const int *Yp, const int *Yi, const cplx *Yx, const int *slack_ids, int nslack,
                  const int *pv, int npv, const int *pq, int npq, const PlanOptions &opt, std::string &msg) {
    P = Plan();
    if (n <= 0 || nslack <= 0) {
        msg = "build_dc_plan: the grid needs at least one bus and one slack bus";
        return NotInitError;
    }
    if (check_ybus(n, Yp, Yi, msg) != NoError) return NotInitError;
    for (int t = 0; t < nslack; ++t)
        if (slack_ids[t] < 0 || slack_ids[t] >= n) { msg = "build_dc_plan: slack id out of range"; return NotInitError; }
    for (int t = 0; t < npv; ++t)
        if (pv[t] < 0 || pv[t] >= n) { msg = "build_dc_plan: PV bus out of range"; return NotInitError; }
    for (int t = 0; t < npq; ++t)
        if (pq[t] < 0 || pq[t] >= n) { msg = "build_dc_plan: PQ bus out of range"; return NotInitError; }
    P.dc = true;
    P.n = n;
    P.nnzY = Yp[n];
    P.Yp.assign(Yp, Yp + n + 1);
    P.Yi.assign(Yi, Yi + P.nnzY);
    P.Yx.assign(Yx, Yx + P.nnzY);
    P.slack0 = slack_ids[0];
    P.slack_ids.assign(slack_ids, slack_ids + nslack);
    P.weights.assign(n, 0.0);
    // BaseDCAlgo::compute_pf (src/powerflow_algorithm/BaseDCAlgo.tpp:55-66): the slacks after
    // the first count as PV (retrieve_pv_with_slack, BaseAlgo.hpp:201-216); the slack buses are
    // the buses neither PV nor PQ (extract_slack_bus_id, BaseAlgo.cpp:143-181); every other bus
    // is an unknown angle, numbered in bus order (fill_mat_bus_id, BaseDCAlgo.tpp:192-201)
    std::vector<char> tagged(n, 0);
    for (int t = 1; t < nslack; ++t) tagged[slack_ids[t]] = 1;
    for (int t = 0; t < npv; ++t) tagged[pv[t]] = 1;
    for (int t = 0; t < npq; ++t) tagged[pq[t]] = 1;
    std::vector<int> id(n, -1);
    int m = 0;
    for (int b = 0; b < n; ++b)
        if (tagged[b]) id[b] = m++;
    if (m == n) { msg = "build_dc_plan: every bus is PV or PQ, there is no slack"; return NotInitError; }
    if (m == 0) { msg = "build_dc_plan: no PV or PQ bus"; return NotInitError; }
    P.m = m;
    make_csr(P);
    // B = Re(Ybus) without the slack rows and columns, Ybus's pattern kept
    // (remove_slack_buses, BaseDCAlgo.tpp:208-232)
    P.Jp.assign(m + 1, 0);
    for (int c = 0; c < n; ++c) {
        if (id[c] < 0) continue;
        for (int p = Yp[c]; p < Yp[c + 1]; ++p)
            if (id[Yi[p]] >= 0) {
                P.Ji.push_back(id[Yi[p]]);
                P.jsrc.push_back(p);
                P.jkind.push_back(0);
                P.jconst.push_back(0.0);
            }
        P.Jp[id[c] + 1] = (int)P.Ji.size();
    }
    for (int c = 0; c < m; ++c) P.Jp[c + 1] = std::max(P.Jp[c + 1], P.Jp[c]);
    std::vector<double> Bx(P.Ji.size());
    for (size_t t = 0; t < Bx.size(); ++t) Bx[t] = Yx[P.jsrc[t]].real();
    PlanOptions o2 = opt;
    o2.dense_tail = false;  // the DC kernel has no dense tail
    const int rc = analyze_lu(P, Bx, o2, msg);
    if (rc != NoError) return rc;
    // bus maps: right-hand side Re(Sbus(b)) at xP[b], angle at xVa[b]
    P.xP.assign(n, -1);
    P.xQ.assign(n, -1);
    P.xVa.assign(n, -1);
    P.xVm.assign(n, -1);
    for (int b = 0; b < n; ++b)
        if (id[b] >= 0) {
            P.xP[b] = P.pinv[id[b]];
            P.xVa[b] = P.qinv[id[b]];
        }
    return NoError;
}

namespace {

// The system of one decoupled half-step: the rows / columns `ids` (grid buses) of a grid-level
// matrix, with their values as the constants of the plan; analysed like a Jacobian and
// factorised on the host by running the refactorisation program's updates in order (the
// operations of a phase are independent, so program order is a valid serial order).
int fdpf_system(Plan &S, int n, const RealCsc &B, const std::vector<int> &ids, const PlanOptions &opt,
                const char *what, std::string &msg, std::vector<double> &lu) {
    S = Plan();
    const int m = (int)ids.size();
    S.m = m;
    std::vector<int> inv(n, -1);
    for (int k = 0; k < m; ++k) inv[ids[k]] = k;
    S.Jp.assign(m + 1, 0);
    std::vector<std::pair<int, double>> col;
    std::vector<double> Bx;
    for (int k = 0; k < m; ++k) {
        const int c = ids[k];
        col.clear();
        for (int p = B.p[c]; p < B.p[c + 1]; ++p)
            if (B.i[p] >= 0 && B.i[p] < n && inv[B.i[p]] >= 0) col.push_back({inv[B.i[p]], B.x[p]});
        std::sort(col.begin(), col.end());
        for (auto &e : col) {
            S.Ji.push_back(e.first);
            S.jsrc.push_back(-1);
            S.jkind.push_back(0);
            S.jconst.push_back(e.second);
            Bx.push_back(e.second);
        }
        S.Jp[k + 1] = (int)S.Ji.size();
    }
    if (m == 0) {
        S.factor.base.assign(1, 0);
        S.backward.base.assign(1, 0);
        S.forward.base.assign(1, 0);
        lu.clear();
        return NoError;
    }
    std::string sub;
    PlanOptions o2 = opt;
    o2.dense_tail = false;  // the fast-decoupled kernel has no dense tail
    const int rc = analyze_lu(S, Bx, o2, sub);
    if (rc != NoError) {
        msg = std::string("build_fdpf_plan: ") + what + ": " + sub;
        return rc;
    }
    lu.assign(S.nnzLU, 0.0);
    for (size_t t = 0; t < S.cpos.size(); ++t) lu[S.cpos[t]] = S.cval[t];
    const int nops = S.factor.nops();
    for (int o = 0; o < nops; ++o) {
        const int *op = &S.factor.ops[4 * (size_t)o];
        if (((unsigned)op[3] >> 28) != 0u) continue;  // substitution pushes and padding
        const int w = op[3] & 0x0fffffff;
        lu[op[0]] -= lu[op[1]] * (lu[op[2]] / lu[w]);
    }
    for (int k = 0; k < m; ++k) {
        const double d = lu[S.dpos[k]];
        if (d == 0.0 || !std::isfinite(d)) {
            msg = std::string("build_fdpf_plan: ") + what + " is singular";
            return SolverFactor;
        }
    }
    return NoError;
}

}  // namespace

int build_fdpf_plan(Plan &P, int n, const int *Yp, const int *Yi, const cplx *Yx, const RealCsc &Bp,
                    const RealCsc &Bpp, const int *slack_ids, int nslack, const double *weights, const int *pv,
                    int npv, const int *pq, int npq, const PlanOptions &opt, std::string &msg) {
    P = Plan();
    if (n <= 0 || nslack <= 0) {
        msg = "build_fdpf_plan: the grid needs at least one bus and one slack bus";
        return NotInitError;
    }
    if (check_ybus(n, Yp, Yi, msg) != NoError) return NotInitError;
    for (const RealCsc *B : {&Bp, &Bpp})
        if (!B->p || !B->i || !B->x || B->p[0] != 0 || B->p[n] < 0) {
            msg = "build_fdpf_plan: B' and B'' must be n x n CSC matrices";
            return NotInitError;
        }
    std::vector<int> role(n, 0);  // 0 none, 1 slack, 2 pv, 3 pq
    for (int t = 0; t < nslack; ++t) {
        if (slack_ids[t] < 0 || slack_ids[t] >= n) { msg = "build_fdpf_plan: slack id out of range"; return NotInitError; }
        role[slack_ids[t]] = 1;
    }
    for (int t = 0; t < npv; ++t) {
        if (pv[t] < 0 || pv[t] >= n || role[pv[t]] != 0) {
            msg = "build_fdpf_plan: a PV bus is out of range, repeated or also a slack";
            return NotInitError;
        }
        role[pv[t]] = 2;
    }
    for (int t = 0; t < npq; ++t) {
        if (pq[t] < 0 || pq[t] >= n || role[pq[t]] != 0) {
            msg = "build_fdpf_plan: a PQ bus is out of range, repeated or also PV / slack";
            return NotInitError;
        }
        role[pq[t]] = 3;
    }
    P.fdpf = true;
    P.factor.base.assign(1, 0);  // no programs of its own: the systems in `sub` carry them
    P.backward.base.assign(1, 0);
    P.forward.base.assign(1, 0);
    P.n = n;
    P.nnzY = Yp[n];
    P.Yp.assign(Yp, Yp + n + 1);
    P.Yi.assign(Yi, Yi + P.nnzY);
    P.Yx.assign(Yx, Yx + P.nnzY);
    P.slack0 = slack_ids[0];
    P.slack_ids.assign(slack_ids, slack_ids + nslack);
    P.weights.assign(weights, weights + n);
    make_csr(P);
    // pvpq = [slacks after the first, pv, pq] (BaseFDPFAlgo.tpp:61-70)
    for (int t = 1; t < nslack; ++t) P.mypv.push_back(slack_ids[t]);
    P.mypv.insert(P.mypv.end(), pv, pv + npv);
    P.pq.assign(pq, pq + npq);
    P.pvpq = P.mypv;
    P.pvpq.insert(P.pvpq.end(), pq, pq + npq);
    P.npv = (int)P.mypv.size();
    P.npq = npq;
    P.npvpq = (int)P.pvpq.size();
    P.sub.resize(2);
    P.sublu.resize(2);
    int rc = fdpf_system(P.sub[0], n, Bp, P.pvpq, opt, "B'", msg, P.sublu[0]);
    if (rc != NoError) return rc;
    rc = fdpf_system(P.sub[1], n, Bpp, P.pq, opt, "B''", msg, P.sublu[1]);
    if (rc != NoError) return rc;
    P.m = P.npvpq + npq;
    // bus maps: P of bus b at xP[b] of the B' right-hand side, its angle step at xVa[b];
    // Q at xQ[b] of the B'' right-hand side, its magnitude step at xVm[b]
    P.xP.assign(n, -1);
    P.xQ.assign(n, -1);
    P.xVa.assign(n, -1);
    P.xVm.assign(n, -1);
    for (int k = 0; k < P.npvpq; ++k) {
        P.xP[P.pvpq[k]] = P.sub[0].pinv[k];
        P.xVa[P.pvpq[k]] = P.sub[0].qinv[k];
    }
    for (int k = 0; k < npq; ++k) {
        P.xQ[pq[k]] = P.sub[1].pinv[k];
        P.xVm[pq[k]] = P.sub[1].qinv[k];
    }
    return NoError;
}

}  // namespace l2g
