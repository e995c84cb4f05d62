// Batched Newton-Raphson over an instance-interleaved value layout: one warp lane per instance.
//
// The kernel of pf_engine.cu gives every instance its own CTA, so each phase of the LU programs
// (one barrier, a dependent chain of loads) serves one instance.  Here a CTA runs 32 instances
// in lock step, one per lane: every LU value, solve-vector entry and bus quantity is stored as 32
// consecutive values, one per instance, so an operation of a phase program is one warp
// instruction over 32 instances and every access is a coalesced 128-byte (FP32) line.  A phase
// costs about what it costs for one instance, and the heavy phases become streaming work on
// HBM.  The programs are the plan's (same operations, same order per written value, so each
// instance computes what the one-CTA kernel computes with its LU in global memory), regrouped so
// that a warp runs whole groups of operations writing one value (TileProgram).
//
// Lanes are refilled as their instances finish: each lane takes jobs from the global counter and
// runs their instances one after the other (chain == 0: every instance starts from its V0).  A
// round does at most one Newton step per lane; the rules are those of the one-CTA kernel
// (BaseNRSingleSlackAlgo::compute_pf, BaseNRSingleSlackAlgo.tpp:12-183; BaseNRAlgo::compute_pf,
// BaseNRAlgo.tpp:14-186): convergence and error codes per instance, and in the mixed form one
// FP64-residual refinement of the step when ||F||_inf < refine_below.
#include "pf_engine.cuh"
#include "pf_device_math.cuh"
#include "pf_plan.hpp"

namespace l2g {
namespace {

constexpr int kLanes = 32;
constexpr int kW = kTileWarps;
static_assert(kW * kLanes == 1024, "the batch-interleaved kernel runs 1024 threads");

enum : int { kFree = 0, kNew = 1, kStep = 2, kDone = 3, kIdle = 4 };

struct TileLanes {
    int inst[kLanes], next[kLanes], end[kLanes], it[kLanes], err[kLanes], state[kLanes], refine[kLanes];
    int novr[kLanes];
    double sa[kLanes];
    int opos[kMaxOverrides][kLanes];
    double2 oval[kMaxOverrides][kLanes];
    double red[kW][kLanes];
    int ired[kW][kLanes];
    int nactive, nstep, nrefine;
    int exhausted;  // a lane found the job list empty
    int handoff;    // the CTA hands its running instances to the one-CTA kernel and stops
    // optional SM cycles per section (A.phase_cycles): mismatch, J fill, refactorisation, forward,
    // backward, refinement residual, update / refill / results, rounds
    unsigned long long pc[kPhaseSlots];
    unsigned long long tmark;
};

// adds the cycles since the last mark to section k (thread 0, when requested)
__device__ __forceinline__ void tile_mark(TileLanes &S, bool on, int k) {
    if (on && threadIdx.x == 0) {
        const unsigned long long t = clock64();
        S.pc[k] += t - S.tmark;
        S.tmark = t;
    }
}

// 32-bit offsets: every slab array has fewer than 2^27 rows
__device__ __forceinline__ unsigned ix(int i, int lane) { return ((unsigned)i << 5) | (unsigned)lane; }

__host__ __device__ __forceinline__ size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

__device__ __forceinline__ double2 ybus_lane(const DevPlan &P, const TileLanes &S, int p, int lane) {
    double2 y = P.Rx[p];
    const int no = S.novr[lane];
    for (int i = 0; i < no; ++i)
        if (S.opos[i][lane] == p) y = S.oval[i][lane];
    return y;
}

// One chunk of a warp: kTileChunk operations, consecutive ones writing one value forming a
// group.  All operands are loaded first (they are final in this phase), then each group
// accumulates in a register and is stored once.  Kinds are 0 (LU update) and 2 (substitution
// push); padding was turned into updates of a per-lane scratch row, so there is no branch.
template <typename LT>
__device__ __forceinline__ void tile_chunk(const int4 *__restrict__ c, LT *lu, LT *x, int lane) {
    int4 o[kTileChunk];
#pragma unroll
    for (int i = 0; i < kTileChunk; ++i) o[i] = __ldg(c + i);
    LT a[kTileChunk], b[kTileChunk], d[kTileChunk], t[kTileChunk];
#pragma unroll
    for (int i = 0; i < kTileChunk; ++i) {
        const bool push = ((unsigned)o[i].w >> 28) != 0u;
        const LT *vsrc = push ? x : lu;
        a[i] = lu[ix(o[i].y, lane)];
        d[i] = lu[ix(o[i].w & 0x0fffffff, lane)];
        b[i] = vsrc[ix(o[i].z, lane)];
        const bool first = i == 0 || o[i].x != o[i - 1].x || o[i].w >> 28 != o[i - 1].w >> 28;
        t[i] = first ? vsrc[ix(o[i].x, lane)] : (LT)0;
    }
    LT acc = (LT)0;
#pragma unroll
    for (int i = 0; i < kTileChunk; ++i) {
        const bool push = ((unsigned)o[i].w >> 28) != 0u;
        const bool first = i == 0 || o[i].x != o[i - 1].x || o[i].w >> 28 != o[i - 1].w >> 28;
        if (first) acc = t[i];
        // LU update by an undivided L entry, or substitution push
        acc -= push ? lu_div(a[i] * b[i], d[i]) : a[i] * lu_div(b[i], d[i]);
        const bool last = i == kTileChunk - 1 || o[i + 1].x != o[i].x || o[i + 1].w >> 28 != o[i].w >> 28;
        if (last) (push ? x : lu)[ix(o[i].x, lane)] = acc;
    }
}

// A program: phase after phase, each warp its chunks, one barrier per phase.  Lanes with act
// false leave their instance's values untouched.
template <typename LT>
__device__ void tile_program(const int4 *__restrict__ ops, const int2 *ph, int nph, LT *lu, LT *x, int lane,
                             int warp, bool act) {
    for (int p = 0; p < nph; ++p) {
        const int2 d = ph[p];
        if (act)
            for (int r = 0; r < d.y; ++r)
                tile_chunk<LT>(ops + ((size_t)d.x + (size_t)r * kW + warp) * kTileChunk, lu, x, lane);
        __syncthreads();
    }
}

template <typename LT, bool REFINE>
__global__ void __launch_bounds__(1024, 1) nr_tile_kernel(const DevPlan P, const BatchArgs A) {
    extern __shared__ __align__(16) int tdyn[];
    __shared__ TileLanes S;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = P.n, m = P.m;
    int2 *phf = reinterpret_cast<int2 *>(tdyn);
    int2 *phb = phf + P.fac_nph;
    int2 *phw = phb + P.bwd_nph;
    for (int i = tid; i < P.fac_nph; i += blockDim.x) phf[i] = make_int2(P.tfac_phase[2 * i], P.tfac_phase[2 * i + 1]);
    for (int i = tid; i < P.bwd_nph; i += blockDim.x) phb[i] = make_int2(P.tbwd_phase[2 * i], P.tbwd_phase[2 * i + 1]);
    for (int i = tid; i < P.fwd_nph; i += blockDim.x) phw[i] = make_int2(P.tfwd_phase[2 * i], P.tfwd_phase[2 * i + 1]);
    unsigned char *q = A.scratch + (size_t)blockIdx.x * (size_t)A.slab_bytes;
    LT *lu = reinterpret_cast<LT *>(q);  // nnzLU rows and a scratch row for padding operations
    q += al256((size_t)(P.nnzLU + 1) * kLanes * sizeof(LT));
    LT *x = reinterpret_cast<LT *>(q);
    q += al256((size_t)m * kLanes * sizeof(LT));
    double *dxg = reinterpret_cast<double *>(q);
    q += al256((size_t)m * kLanes * 8);
    double2 *V = reinterpret_cast<double2 *>(q);
    q += al256((size_t)n * kLanes * 16);
    double2 *Ib = reinterpret_cast<double2 *>(q);
    q += al256((size_t)n * kLanes * 16);
    double2 *Fb = reinterpret_cast<double2 *>(q);
    q += al256((size_t)n * kLanes * 16);
    double *Vm = reinterpret_cast<double *>(q);
    q += al256((size_t)n * kLanes * 8);
    double *Va = reinterpret_cast<double *>(q);
    q += al256((size_t)n * kLanes * 8);
    double2 *dV = reinterpret_cast<double2 *>(q);  // the refinement's voltage step
    const bool prof = A.phase_cycles != nullptr;
    if (tid == 0) {
        S.exhausted = 0;
        S.handoff = 0;
        for (int k = 0; k < kPhaseSlots; ++k) S.pc[k] = 0;
        S.tmark = clock64();
    }
    if (tid < kLanes) {
        S.state[tid] = tid < A.tile_lanes ? kFree : kIdle;
        S.next[tid] = S.end[tid] = 0;
        S.inst[tid] = 0;
        S.novr[tid] = 0;
        S.refine[tid] = 0;
    }
    __syncthreads();
    for (;;) {
        // ---- refill: finished lanes take the next instance of their job, or a new job
        tile_mark(S, prof, 6);
        if (prof && tid == 0) S.pc[7] += 1;
        if (warp == 0) {
            int st = S.state[lane];
            int lane_exh = 0;
            if (st == kFree || st == kDone) {
                st = kIdle;
                while (S.next[lane] >= S.end[lane]) {
                    const int j = atomicAdd(A.job_counter, 1);
                    if (j >= A.njobs) {
                        lane_exh = 1;
                        break;
                    }
                    S.next[lane] = A.job_first[j];
                    S.end[lane] = A.job_first[j] + A.job_count[j];
                }
                if (S.next[lane] < S.end[lane]) {
                    const int inst = S.next[lane]++;
                    S.inst[lane] = inst;
                    S.it[lane] = 0;
                    S.err[lane] = 0;
                    st = kNew;
                    int k0 = 0, k1 = 0;
                    if (A.ovr_ptr) {
                        k0 = A.ovr_ptr[inst];
                        k1 = A.ovr_ptr[inst + 1];
                    }
                    if (k1 - k0 > kMaxOverrides) {
                        S.novr[lane] = 0;
                        S.err[lane] = 8;  // NotInitError: more overrides than staged, not computed
                    } else {
                        S.novr[lane] = k1 - k0;
                        for (int i = 0; i < k1 - k0; ++i) {
                            S.opos[i][lane] = A.ovr_pos[k0 + i];
                            S.oval[i][lane] = A.ovr_val[k0 + i];
                        }
                    }
                }
            }
            S.state[lane] = st;
            const unsigned act = __ballot_sync(0xffffffffu, st == kNew || st == kStep);
            const bool exh = __any_sync(0xffffffffu, lane_exh != 0);
            if (lane == 0) {
                S.nactive = __popc(act);
                if (exh) S.exhausted = 1;
                // stragglers: with the jobs exhausted, a round costs about as much for a few lanes
                // as for all of them, so the last few instances continue on the one-CTA kernel
                // (single slack only: there the Newton state is V alone)
                S.handoff = A.hand_list != nullptr && !P.distributed && S.exhausted && S.nactive > 0 &&
                            S.nactive <= A.hand_lanes;
            }
        }
        __syncthreads();
        if (S.nactive == 0) break;
        if (S.handoff) {
            // the state of every running lane into its output row: V (the start voltages for a lane
            // that has not started), the iterations taken so far; the instance joins the list
            const int st = S.state[lane];
            const bool run = st == kNew || st == kStep;
            const int inst = S.inst[lane];
            if (run) {
                double2 *vo = out_row(A, inst, n);
                const double2 *v0 = A.V0 + (long long)inst * A.v0_stride;
                for (int r = warp; r < n; r += kW) vo[r] = st == kNew ? v0[r] : V[ix(r, lane)];
            }
            if (warp == 0 && run) {
                A.iters[inst] = S.it[lane];
                A.errs[inst] = 0;
                A.hand_list[atomicAdd(A.hand_count, 1)] = inst;
            }
            break;
        }
        const bool fresh = S.state[lane] == kNew;
        const int inst = S.inst[lane];
        const double2 *Sb = A.Sbus + (long long)inst * A.sbus_stride;
        // ---- start voltages of the new lanes; slack_absorbed of a distributed slack
        {
            double ls = 0.0;
            if (fresh) {
                const double2 *v0 = A.V0 + (long long)inst * A.v0_stride;
                for (int r = warp; r < n; r += kW) {
                    const double2 v = v0[r];
                    V[ix(r, lane)] = v;
                    Vm[ix(r, lane)] = cabs2(v);
                    Va[ix(r, lane)] = atan2(v.y, v.x);
                    ls += Sb[r].x;
                }
            }
            S.red[warp][lane] = ls;
            __syncthreads();
            if (warp == 0 && fresh) {
                double t = 0.0;
                if (P.distributed)
                    for (int w = 0; w < kW; ++w) t += S.red[w][lane];
                S.sa[lane] = t;
            }
            __syncthreads();
        }
        // ---- mismatch F = V conj(Ybus V) - Sbus (+ slack term): Ibus, F, right-hand side, ||F||
        {
            const int st = S.state[lane];
            const bool on = st == kNew || st == kStep;
            double lmax = 0.0;
            int lbad = 0;
            if (on) {
                const double sa = S.sa[lane];
                for (int r = warp; r < n; r += kW) {
                    double2 s = make_double2(0.0, 0.0);
                    const int p1 = P.Rp[r + 1];
                    for (int p = P.Rp[r]; p < p1; ++p) {
                        const double2 y = ybus_lane(P, S, p, lane);
                        const double2 vv = V[ix(P.Rj[p], lane)];
                        s.x += y.x * vv.x - y.y * vv.y;
                        s.y += y.x * vv.y + y.y * vv.x;
                    }
                    Ib[ix(r, lane)] = s;
                    const double2 vr = V[ix(r, lane)];
                    const double2 sb = Sb[r];
                    double mr = vr.x * s.x + vr.y * s.y - sb.x;
                    const double mi = vr.y * s.x - vr.x * s.y - sb.y;
                    if (P.distributed) mr += sa * P.w[r];
                    Fb[ix(r, lane)] = make_double2(mr, mi);
                    const int ip = P.xP[r], iq = P.xQ[r];
                    if (ip >= 0) {
                        x[ix(ip, lane)] = (LT)mr;
                        lmax = fmax(lmax, fabs(mr));
                        lbad |= !isfinite(mr);
                    }
                    if (iq >= 0) {
                        x[ix(iq, lane)] = (LT)mi;
                        lmax = fmax(lmax, fabs(mi));
                        lbad |= !isfinite(mi);
                    }
                }
            }
            S.red[warp][lane] = lmax;
            S.ired[warp][lane] = lbad;
        }
        __syncthreads();
        tile_mark(S, prof, 0);
        // ---- per-instance decisions
        if (warp == 0) {
            int st = S.state[lane];
            double norm = 0.0;
            int bad = 0;
            for (int w = 0; w < kW; ++w) {
                norm = fmax(norm, S.red[w][lane]);
                bad |= S.ired[w][lane];
            }
            if (st == kNew) {
                if (S.err[lane] != 0 || (!bad && norm < A.tol)) {
                    st = kDone;
                } else if (A.max_iter <= 0) {
                    S.err[lane] = 2;  // TooManyIterations
                    st = kDone;
                } else {
                    st = kStep;
                }
            } else if (st == kStep) {
                if (bad) {
                    S.err[lane] = 3;  // InifiniteValue
                    st = kDone;
                } else if (norm < A.tol) {
                    st = kDone;
                } else if (S.it[lane] >= A.max_iter) {
                    S.err[lane] = 2;  // TooManyIterations
                    st = kDone;
                }
            }
            const int rf = (REFINE && st == kStep && norm < A.refine_below) ? 1 : 0;
            S.refine[lane] = rf;
            if (st == kStep) S.it[lane] += 1;
            S.state[lane] = st;
            const unsigned sm = __ballot_sync(0xffffffffu, st == kStep);
            const unsigned rm = __ballot_sync(0xffffffffu, rf != 0);
            if (lane == 0) {
                S.nstep = __popc(sm);
                S.nrefine = __popc(rm);
            }
        }
        __syncthreads();
        if (S.nstep > 0) {
            const bool step = S.state[lane] == kStep;
            // ---- Jacobian values (dS/dVa, dS/dVm) into the LU array
            if (step) {
                for (int p = warp; p < P.nnzY; p += kW) {
                    const int r = P.Rrow[p], c = P.Rj[p];
                    double dvar, dvai;
                    double2 dvm;
                    dsbus(ybus_lane(P, S, p, lane), V[ix(r, lane)], V[ix(c, lane)], r == c,
                          r == c ? Ib[ix(r, lane)] : make_double2(0.0, 0.0), dvar, dvai, dvm);
                    const int4 t = P.ytarget[p];
                    if (t.x >= 0) lu[ix(t.x, lane)] = (LT)dvar;
                    if (t.y >= 0) lu[ix(t.y, lane)] = (LT)dvai;
                    if (t.z >= 0) lu[ix(t.z, lane)] = (LT)dvm.x;
                    if (t.w >= 0) lu[ix(t.w, lane)] = (LT)dvm.y;
                }
                for (int i = warp; i < P.nfill; i += kW) lu[ix(P.fillpos[i], lane)] = (LT)0;
                for (int i = warp; i < P.nconst; i += kW) lu[ix(P.cpos[i], lane)] = (LT)P.cval[i];
            }
            __syncthreads();
            tile_mark(S, prof, 1);
            // ---- refactorisation with the forward substitution of F fused in
            tile_program<LT>(P.tfac_ops, phf, P.fac_nph, lu, x, lane, warp, step);
            tile_mark(S, prof, 2);
            {
                int zero = 0;
                if (step)
                    for (int k = warp; k < m; k += kW) zero |= lu[ix(P.dpos[k], lane)] == (LT)0;
                S.ired[warp][lane] = zero;
            }
            __syncthreads();
            if (warp == 0 && step) {
                int zero = 0;
                for (int w = 0; w < kW; ++w) zero |= S.ired[w][lane];
                if (zero) {
                    S.err[lane] = 6;  // SolverReFactor: a zero pivot, the step is not taken
                    S.state[lane] = kDone;
                }
            }
            __syncthreads();
            const bool solve = S.state[lane] == kStep;
            // ---- backward substitution and the pivot scaling
            tile_mark(S, prof, 6);
            tile_program<LT>(P.tbwd_ops, phb, P.bwd_nph, lu, x, lane, warp, solve);
            if (solve)
                for (int k = warp; k < m; k += kW) x[ix(k, lane)] = lu_div(x[ix(k, lane)], lu[ix(P.dpos[k], lane)]);
            __syncthreads();
            tile_mark(S, prof, 4);
            const bool refine = solve && S.refine[lane] != 0;
            if (REFINE && S.nrefine > 0) {
                // ---- refinement against the FP64 Jacobian: rhs = F - J dx, solved again
                if (refine)
                    for (int k = warp; k < m; k += kW) dxg[ix(k, lane)] = (double)x[ix(k, lane)];
                __syncthreads();
                // J dx = dV conj(I) + V conj(Y dV), dV = V / |V| dVm + j V dVa: the linearisation
                // of S(V) = V conj(Y V) that the Jacobian holds (as the one-CTA kernel forms it)
                if (refine)
                    for (int b = warp; b < n; b += kW) {
                        const int ia = P.xVa[b], im = P.xVm[b];
                        const double2 v = V[ix(b, lane)];
                        const double dA = ia >= 0 ? dxg[ix(ia, lane)] : 0.0;
                        const double dM = im >= 0 ? dxg[ix(im, lane)] / cabs2(v) : 0.0;
                        dV[ix(b, lane)] = make_double2(v.x * dM - v.y * dA, v.y * dM + v.x * dA);
                    }
                __syncthreads();
                if (refine)
                    for (int r = warp; r < n; r += kW) {
                        const int ip = P.xP[r], iq = P.xQ[r];
                        if (ip < 0 && iq < 0) continue;
                        double2 yd = make_double2(0.0, 0.0);
                        const int p1 = P.Rp[r + 1];
                        for (int p = P.Rp[r]; p < p1; ++p) {
                            const double2 y = ybus_lane(P, S, p, lane), d = dV[ix(P.Rj[p], lane)];
                            yd.x += y.x * d.x - y.y * d.y;
                            yd.y += y.x * d.y + y.y * d.x;
                        }
                        const double2 vr = V[ix(r, lane)], dvr = dV[ix(r, lane)], ir = Ib[ix(r, lane)];
                        double jP = dvr.x * ir.x + dvr.y * ir.y + (vr.x * yd.x + vr.y * yd.y);
                        const double jQ = dvr.y * ir.x - dvr.x * ir.y + (vr.y * yd.x - vr.x * yd.y);
                        if (P.distributed && ip >= 0) jP += P.wJ[r] * dxg[ix(P.xSlack, lane)];
                        const double2 F = Fb[ix(r, lane)];
                        if (ip >= 0) x[ix(ip, lane)] = (LT)(F.x - jP);
                        if (iq >= 0) x[ix(iq, lane)] = (LT)(F.y - jQ);
                    }
                __syncthreads();
                tile_mark(S, prof, 5);
                tile_program<LT>(P.tfwd_ops, phw, P.fwd_nph, lu, x, lane, warp, refine);
                tile_mark(S, prof, 3);
                tile_program<LT>(P.tbwd_ops, phb, P.bwd_nph, lu, x, lane, warp, refine);
                if (refine)
                    for (int k = warp; k < m; k += kW)
                        x[ix(k, lane)] = lu_div(x[ix(k, lane)], lu[ix(P.dpos[k], lane)]);
                __syncthreads();
                tile_mark(S, prof, 4);
            }
            // ---- voltage update
            double lmin = 1.0;
            if (solve)
                for (int r = warp; r < n; r += kW) {
                    // Vm and Va as updated, re-derived from V only where that changes them (as
                    // in the one-CTA kernel's voltage_update)
                    double vm = Vm[ix(r, lane)], va = Va[ix(r, lane)];
                    const int ia = P.xVa[r], im = P.xVm[r];
                    if (ia >= 0) va -= refine ? dxg[ix(ia, lane)] + (double)x[ix(ia, lane)] : (double)x[ix(ia, lane)];
                    if (im >= 0) vm -= refine ? dxg[ix(im, lane)] + (double)x[ix(im, lane)] : (double)x[ix(im, lane)];
                    double sn, cs;
                    sincos(va, &sn, &cs);
                    const double2 v = make_double2(vm * cs, vm * sn);
                    V[ix(r, lane)] = v;
                    lmin = fmin(lmin, vm);
                    if (!P.distributed && !(vm >= 0.0 && fabs(va) <= kPi)) {
                        vm = cabs2(v);
                        va = atan2(v.y, v.x);
                    }
                    Vm[ix(r, lane)] = vm;
                    Va[ix(r, lane)] = va;
                }
            if (P.distributed) {
                S.red[warp][lane] = lmin;
                __syncthreads();
                if (warp == 0) {
                    double vmin = 1.0;
                    for (int w = 0; w < kW; ++w) vmin = fmin(vmin, S.red[w][lane]);
                    S.ired[0][lane] = solve && vmin < 0.0;
                    if (solve) {
                        const int k = P.xSlack;
                        S.sa[lane] -= refine ? dxg[ix(k, lane)] + (double)x[ix(k, lane)] : (double)x[ix(k, lane)];
                    }
                }
                __syncthreads();
                if (S.ired[0][lane])
                    for (int r = warp; r < n; r += kW) {
                        const double2 v = V[ix(r, lane)];
                        Vm[ix(r, lane)] = cabs2(v);
                        Va[ix(r, lane)] = atan2(v.y, v.x);
                    }
            }
        }
        // ---- results of the instances that finished in this round
        if (S.state[lane] == kDone) {
            double2 *vo = out_row(A, inst, n);
            const bool zero = A.zero_failed && S.err[lane] != 0;
            for (int r = warp; r < n; r += kW) vo[r] = zero ? make_double2(0.0, 0.0) : V[ix(r, lane)];
            if (warp == 0) {
                A.iters[inst] = S.it[lane];
                A.errs[inst] = S.err[lane];
                // mixed form: an instance that failed in FP32 is solved again in FP64 afterwards
                if (A.fb_list != nullptr && S.err[lane] != 0) A.fb_list[atomicAdd(A.fb_count, 1)] = inst;
            }
        }
        __syncthreads();
    }
    if (prof && tid == 0) {
        tile_mark(S, prof, 6);
        for (int k = 0; k < kPhaseSlots; ++k) A.phase_cycles[(size_t)blockIdx.x * kPhaseSlots + k] = S.pc[k];
    }
}

template <typename LT, bool RF>
cudaError_t launch_tile_variant(const DevPlan &P, const BatchArgs &A, int grid, size_t smem, cudaStream_t st) {
    cudaError_t e = allow_max_smem(reinterpret_cast<const void *>(nr_tile_kernel<LT, RF>));
    if (e != cudaSuccess) return e;
    nr_tile_kernel<LT, RF><<<grid, kW * kLanes, smem, st>>>(P, A);
    return cudaGetLastError();
}

}  // namespace

size_t tile_slab_bytes(const DevPlan &P, int lu_bytes) {
    const size_t L = kLanes;
    return al256((size_t)(P.nnzLU + 1) * L * lu_bytes) + al256((size_t)P.m * L * lu_bytes) + al256((size_t)P.m * L * 8) +
           4 * al256((size_t)P.n * L * 16) + 2 * al256((size_t)P.n * L * 8);
}

size_t tile_smem_bytes(const DevPlan &P) { return (size_t)(P.fac_nph + P.bwd_nph + P.fwd_nph) * sizeof(int2); }

cudaError_t launch_nr_tile(const DevPlan &P, const BatchArgs &A, int precision, int grid, cudaStream_t stream) {
    const size_t smem = tile_smem_bytes(P);
    if (precision == 0) return launch_tile_variant<double, false>(P, A, grid, smem, stream);
    if (A.refine) return launch_tile_variant<float, true>(P, A, grid, smem, stream);
    return launch_tile_variant<float, false>(P, A, grid, smem, stream);
}

}  // namespace l2g
