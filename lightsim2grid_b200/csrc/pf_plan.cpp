// Host-side symbolic analysis: Jacobian pattern, ordering, first factorisation, schedules.
#include "pf_plan.hpp"

#include <algorithm>
#include <cmath>
#include <sstream>

namespace l2g {

namespace {

// -------------------------------------------------------------------------------------
// Minimum-degree ordering on the symmetric pattern of A + A^T.
//
// Explicit elimination graph (Rose 1972; Tinney & Walker scheme 2): eliminating v joins
// its neighbours into a clique.  Degrees are kept in bucket lists so that the next
// minimum is found in O(1); ties go to the most recently touched node of the bucket.
// -------------------------------------------------------------------------------------
std::vector<int> minimum_degree(int m, const std::vector<int> &Ap, const std::vector<int> &Ai) {
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
    for (int k = 0; k < m; ++k) {
        while (mindeg <= m && head[mindeg] < 0) ++mindeg;
        int v = head[mindeg];
        unlink(v);
        alive[v] = 0;
        order.push_back(v);
        const std::vector<int> nb = adj[v];
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

int lanes_for(int maxlen) {
    if (maxlen <= 2) return 1;
    if (maxlen <= 4) return 2;
    if (maxlen <= 8) return 4;
    if (maxlen <= 16) return 8;
    if (maxlen <= 32) return 16;
    return 32;
}

// Groups items by level: each level becomes a wide group, except runs of consecutive
// levels with at most `chain_max` items, which become one chain group.
void make_groups(const std::vector<int> &level, const std::vector<int> &itemlen, int chain_max,
                 std::vector<int> &order, std::vector<LevelGroup> &groups, int &nlevels, bool solve) {
    int m = (int)level.size();
    nlevels = 0;
    for (int v : level) nlevels = std::max(nlevels, v + 1);
    std::vector<int> cnt(nlevels + 1, 0);
    for (int v : level) cnt[v + 1]++;
    for (int l = 0; l < nlevels; ++l) cnt[l + 1] += cnt[l];
    order.assign(m, 0);
    std::vector<int> fillp(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < m; ++i) order[fillp[level[i]]++] = i;
    // within a level, longest items first (better balance of the round-robin)
    for (int l = 0; l < nlevels; ++l)
        std::stable_sort(order.begin() + cnt[l], order.begin() + cnt[l + 1],
                         [&](int a, int b) { return itemlen[a] > itemlen[b]; });
    groups.clear();
    int l = 0;
    while (l < nlevels) {
        int sz = cnt[l + 1] - cnt[l];
        if (sz <= chain_max) {
            int l2 = l;
            int maxlen = 0;
            while (l2 < nlevels && cnt[l2 + 1] - cnt[l2] <= chain_max) {
                for (int t = cnt[l2]; t < cnt[l2 + 1]; ++t) maxlen = std::max(maxlen, itemlen[order[t]]);
                ++l2;
            }
            groups.push_back({cnt[l], cnt[l2], 1, solve ? lanes_for(maxlen) : 32});
            l = l2;
        } else {
            int maxlen = 0;
            for (int t = cnt[l]; t < cnt[l + 1]; ++t) maxlen = std::max(maxlen, itemlen[order[t]]);
            groups.push_back({cnt[l], cnt[l + 1], 0, solve ? lanes_for(maxlen) : 32});
            ++l;
        }
    }
}

}  // namespace

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

    // CSR copy
    P.Rp.assign(n + 1, 0);
    for (int p = 0; p < P.nnzY; ++p) P.Rp[P.Yi[p] + 1]++;
    for (int r = 0; r < n; ++r) P.Rp[r + 1] += P.Rp[r];
    P.Rj.assign(P.nnzY, 0);
    P.Rrow.assign(P.nnzY, 0);
    P.csr_of_csc.assign(P.nnzY, 0);
    P.Rx.assign(P.nnzY, 0.0);
    {
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

    // ---------------------------------------------------------------- ordering
    P.q = minimum_degree(m, P.Jp, P.Ji);
    P.qinv.assign(m, 0);
    for (int k = 0; k < m; ++k) P.qinv[P.q[k]] = k;

    // ---------------------------------------------------------------- first factorisation
    std::vector<cplx> Vinit(V0, V0 + n);
    std::vector<double> Jx;
    host_jacobian(P, P.Yx.data(), Vinit.data(), Jx);
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
                err << "build_plan: the first Jacobian is singular (step " << k << ")";
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

    // ---------------------------------------------------------------- refactorisation schedule
    // levels: a pivot can be applied once every pivot updating its column is done
    std::vector<int> level(m, 0);
    P.flops_refactor = 0;
    for (int k = 0; k < m; ++k) {
        int lv = 0;
        for (int c : Ucols[k]) lv = std::max(lv, level[c] + 1);
        level[k] = lv;
        for (int c : Ucols[k]) P.flops_refactor += P.lcount[c];
    }
    P.colleve = level;
    int nlev = 0;
    for (int v : level) nlev = std::max(nlev, v + 1);
    P.levels_refactor = nlev;
    // U row lists: for pivot c, the columns j > c with U(c, j) != 0 and the position of U(c, j)
    std::vector<std::vector<std::pair<int, int>>> urows(m);
    for (int k = 0; k < m; ++k)
        for (size_t t = 0; t < Ucols[k].size(); ++t) urows[Ucols[k][t]].push_back({k, P.colstart[k] + (int)t});
    std::vector<std::vector<int>> bylevel(nlev);
    for (int k = 0; k < m; ++k) bylevel[level[k]].push_back(k);
    std::vector<int> rowpos(m, -1);
    std::vector<uint64_t> used(P.nnzLU, 0);  // phases of the current level writing an entry
    std::vector<int> used_level(P.nnzLU, -1);
    std::vector<int> pend_div;               // pivots whose divisions are pending
    for (int l = 0; l < nlev; ++l) {
        // the groups of this level
        struct G { int c, j, upos; };
        std::vector<G> gs;
        for (int c : bylevel[l])
            for (auto &e : urows[c]) gs.push_back({c, e.first, e.second});
        // greedy colouring into conflict-free phases (first fit in group order)
        std::vector<std::vector<int>> ph_groups;
        std::vector<std::vector<int>> gdst(gs.size());
        for (size_t g = 0; g < gs.size(); ++g) {
            const int c = gs[g].c, j = gs[g].j;
            for (int p = P.colstart[j]; p < P.colstart[j + 1]; ++p) rowpos[P.Urow_k[p]] = p;
            for (int s = 0; s < P.lcount[c]; ++s) {
                int d = rowpos[Lrows[c][s]];
                if (d < 0) {
                    msg = "build_plan: internal error, LU pattern is not closed";
                    return SolverAnalyze;
                }
                gdst[g].push_back(d);
            }
            for (int p = P.colstart[j]; p < P.colstart[j + 1]; ++p) rowpos[P.Urow_k[p]] = -1;
            uint64_t busy = 0;
            for (int d : gdst[g]) {
                if (used_level[d] != l) {
                    used_level[d] = l;
                    used[d] = 0;
                }
                busy |= used[d];
            }
            int ph = 0;
            while (ph < 64 && ((busy >> ph) & 1u)) ++ph;
            if (ph == 64) {
                msg = "build_plan: more than 64 conflicting update phases in one level";
                return SolverAnalyze;
            }
            for (int d : gdst[g]) used[d] |= (uint64_t)1 << ph;
            if ((int)ph_groups.size() <= ph) ph_groups.resize(ph + 1);
            ph_groups[ph].push_back((int)g);
        }
        if (ph_groups.empty()) ph_groups.resize(1);  // a level with no updates still divides
        for (size_t ph = 0; ph < ph_groups.size(); ++ph) {
            Plan::Phase Q;
            Q.gbeg = (int)P.grp_lstart.size();
            int maxlc = 0;
            // longest groups first: better balance of the round-robin
            std::stable_sort(ph_groups[ph].begin(), ph_groups[ph].end(), [&](int a, int b) {
                return P.lcount[gs[a].c] > P.lcount[gs[b].c];
            });
            for (int g : ph_groups[ph]) {
                const int c = gs[g].c;
                P.grp_lstart.push_back(P.lstart[c]);
                P.grp_lcount.push_back(P.lcount[c]);
                P.grp_upos.push_back(gs[g].upos);
                P.grp_dpos.push_back(P.dpos[c]);
                P.grp_dst.push_back((int)P.dst.size());
                P.dst.insert(P.dst.end(), gdst[g].begin(), gdst[g].end());
                maxlc = std::max(maxlc, P.lcount[c]);
            }
            Q.gend = (int)P.grp_lstart.size();
            Q.dbeg = (int)P.div_pos.size();
            if (ph == 0) {
                for (int c : pend_div)
                    for (int t = 0; t < P.lcount[c]; ++t) {
                        P.div_pos.push_back(P.lstart[c] + t);
                        P.div_dpos.push_back(P.dpos[c]);
                    }
                pend_div.clear();
            }
            Q.dend = (int)P.div_pos.size();
            Q.lanes = lanes_for(maxlc);
            P.phases.push_back(Q);
        }
        pend_div = bylevel[l];
    }
    {
        // trailing phase: divisions of the last level, and the pivot check of every column
        Plan::Phase Q;
        Q.gbeg = Q.gend = (int)P.grp_lstart.size();
        Q.dbeg = (int)P.div_pos.size();
        for (int c : pend_div)
            for (int t = 0; t < P.lcount[c]; ++t) {
                P.div_pos.push_back(P.lstart[c] + t);
                P.div_dpos.push_back(P.dpos[c]);
            }
        Q.dend = (int)P.div_pos.size();
        Q.lanes = 1;
        P.phases.push_back(Q);
    }

    // ---------------------------------------------------------------- triangular solves
    {
        std::vector<std::vector<std::pair<int, int>>> lr(m), ur(m);
        for (int k = 0; k < m; ++k) {
            for (int t = 0; t < P.lcount[k]; ++t) lr[Lrows[k][t]].push_back({k, P.lstart[k] + t});
            for (size_t t = 0; t < Ucols[k].size(); ++t) ur[Ucols[k][t]].push_back({k, P.colstart[k] + (int)t});
        }
        P.lrow_ptr.assign(m + 1, 0);
        P.urow_ptr.assign(m + 1, 0);
        std::vector<int> lvL(m, 0), lvU(m, 0), lenL(m), lenU(m);
        for (int i = 0; i < m; ++i) {
            int lv = 0;
            for (auto &e : lr[i]) {
                P.lrow_col.push_back(e.first);
                P.lrow_pos.push_back(e.second);
                lv = std::max(lv, lvL[e.first] + 1);
            }
            lvL[i] = lv;
            lenL[i] = (int)lr[i].size();
            P.lrow_ptr[i + 1] = (int)P.lrow_col.size();
        }
        for (int i = 0; i < m; ++i) {
            for (auto &e : ur[i]) {
                P.urow_col.push_back(e.first);
                P.urow_pos.push_back(e.second);
            }
            lenU[i] = (int)ur[i].size();
            P.urow_ptr[i + 1] = (int)P.urow_col.size();
        }
        for (int i = m - 1; i >= 0; --i) {
            int lv = 0;
            for (auto &e : ur[i]) lv = std::max(lv, lvU[e.first] + 1);
            lvU[i] = lv;
        }
        make_groups(lvL, lenL, opt.chain_max_items, P.fwd_order, P.fwd_groups, P.levels_fwd, true);
        make_groups(lvU, lenU, opt.chain_max_items, P.bwd_order, P.bwd_groups, P.levels_bwd, true);
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

}  // namespace l2g
