// Batched AC Newton-Raphson on the GPU: one persistent kernel, one CTA per instance.
//
// Each CTA takes jobs (an instance, or a chain of time-series steps) from a global
// counter and runs the whole Newton loop of the reference's compute_pf for them:
//   mismatch   F = V .* conj(Ybus V) - Sbus (+ slack term)     BaseAlgo.cpp:30-118
//   J fill     dS/dVm, dS/dVa scattered into the LU array      BaseNRAlgo.tpp:202-260,
//                                                              BaseNRSingleSlackAlgo.tpp:449-490
//   refactor   LU with the plan's fixed pivots                 (KLUSolver.cpp:47-59 contract)
//   solve      forward / backward substitution                 (KLUSolver.cpp:61-69 contract)
//   update     Va, Vm, V and the convergence test              BaseNRSingleSlackAlgo.tpp:129-162,
//                                                              BaseNRAlgo.tpp:136-167
// The refactorisation (right-looking, by elimination level, with the forward substitution
// of the right-hand side fused in) and the substitutions run as phase programs: flat lists
// of independent operations, coloured on the host into conflict-free phases, one barrier
// per phase, no atomics -- the result is deterministic.  LU values live in shared memory
// when they fit, else in the CTA's global slab (L2 resident).  The mixed form (FP32 LU)
// refines the Newton steps taken close to the solution once against the FP64 Jacobian,
// computed on the fly from dS/dV (the correction solve is skipped when the FP64 residual is
// already below a hundredth of the tolerance).
#include "pf_engine.cuh"
#include "pf_device_math.cuh"

#include <mutex>
#include <set>
#include <utility>

namespace l2g {

namespace {



struct Shared {
    double red[32];  // block reductions; the dense tail's backward substitution (one panel's values)
    int ired[32];
    unsigned long long pc[kPhaseSlots];  // per-phase SM cycles (thread 0, when profiled)
    int opos[kMaxOverrides];
    double2 oval[kMaxOverrides];
    int novr;
    int job;
    int piv_err;
    int job_failed;
    double slack_absorbed;
};

// load with acquire semantics at GPU scope: the job ring entries and segments written before the
// tail (by the host's copies, in stream order) are seen after it
__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Request loop: claims the next published job of the ring (compare-and-swap on the head, so a
// CTA never holds a job that is not there yet) into *job and returns its index, or -1 when the
// launch is closing and the ring is empty.  After idle_polls polls of an empty ring the CTA closes
// the launch (every CTA then leaves at its next empty poll), so the wait is bounded.  A function of
// its own: its registers do not add to the solver's.
__device__ __noinline__ int claim_queue_job(const QueueJob *jobs, int cap, int *head, const int *tail, int *closing,
                                            int idle_polls, QueueJob *job) {
    for (int polls = 0;;) {
        const int t = ld_acquire_gpu(tail);
        const int h = *reinterpret_cast<volatile int *>(head);
        if (h < t) {
            if (atomicCAS(head, h, h + 1) == h) {
                const QueueJob *e = jobs + (h % cap);
                *job = QueueJob{__ldcg(&e->slot), __ldcg(&e->first), __ldcg(&e->count), __ldcg(&e->req)};
                return h;
            }
            continue;  // another CTA took it: look again
        }
        if (*reinterpret_cast<volatile int *>(closing)) return -1;
        if (++polls > idle_polls) {
            atomicExch(closing, 1);
            return -1;
        }
        __nanosleep(500);
    }
}

// Request loop: the job's rows, iterations and errors (mapped host memory) are made visible before
// its instances are added to the slot's completion count.
__device__ __noinline__ void signal_queue_job(int *done, int slot, int count) {
    __threadfence_system();
    atomicAdd_system(done + slot, count);
}

// block-wide max of |F| and "any non-finite" flag; every thread receives the result
__device__ __forceinline__ void block_norm(Shared &S, double lmax, int lbad, double &norm, int &bad) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
        lbad |= __shfl_xor_sync(0xffffffffu, lbad, o);
    }
    __syncthreads();
    if (lane == 0) {
        S.red[warp] = lmax;
        S.ired[warp] = lbad;
    }
    __syncthreads();
    double r = 0.0;
    int b = 0;
    for (int w = 0; w < nw; ++w) {
        r = fmax(r, S.red[w]);
        b |= S.ired[w];
    }
    norm = r;
    bad = b;
}

__device__ __forceinline__ double block_min(Shared &S, double v) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) S.red[warp] = v;
    __syncthreads();
    double r = S.red[0];
    for (int w = 1; w < nw; ++w) r = fmin(r, S.red[w]);
    return r;
}

__device__ __forceinline__ double block_sum(Shared &S, double v) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) S.red[warp] = v;
    __syncthreads();
    double r = 0.0;
    for (int w = 0; w < nw; ++w) r += S.red[w];
    return r;
}

__device__ __forceinline__ double2 ybus_value(const DevPlan &P, const Shared &S, int p) {
    double2 y = P.Rx[p];
    for (int i = 0; i < S.novr; ++i)
        if (S.opos[i] == p) y = S.oval[i];
    return y;
}


// (Ybus V)[r], over the row's entries in column order
__device__ __forceinline__ double2 ybus_row_product(const DevPlan &P, const Shared &S, const double2 *__restrict__ V,
                                                    int r) {
    double2 s = make_double2(0.0, 0.0);
    const int p0 = P.Rp[r], p1 = P.Rp[r + 1];
    for (int p = p0; p < p1; p += 4) {
        // indices first, then values: the loads of four entries are in flight together
        int c[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) c[u] = p + u < p1 ? P.Rj[p + u] : -1;
        double2 y[4], vv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            y[u] = c[u] >= 0 ? ybus_value(P, S, p + u) : make_double2(0.0, 0.0);
            vv[u] = c[u] >= 0 ? V[c[u]] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            s.x += y[u].x * vv[u].x - y[u].y * vv[u].y;
            s.y += y[u].x * vv[u].y + y[u].y * vv[u].x;
        }
    }
    return s;
}

// F at V: writes Ibus, the FP64 mismatch per bus and the permuted right-hand side x;
// returns ||F||_inf and a non-finite flag to every thread.
template <typename XT>
__device__ void mismatch(const DevPlan &P, Shared &S, const double2 *__restrict__ V, double2 *__restrict__ Ibus,
                         double2 *__restrict__ Fbus, const double2 *__restrict__ Sbus, XT *x, double &norm,
                         int &bad) {
    double lmax = 0.0;
    int lbad = 0;
    const double sa = S.slack_absorbed;
    for (int r = threadIdx.x; r < P.n; r += blockDim.x) {
        // the row's own loads are issued before the row product (they do not depend on it)
        const double2 sb = __ldcg(Sbus + r);
        const int ip = P.xP[r], iq = P.xQ[r];
        const double2 s = ybus_row_product(P, S, V, r);
        Ibus[r] = s;
        const double2 vr = V[r];
        double mr = vr.x * s.x + vr.y * s.y - sb.x;  // V * conj(I) - S
        const double mi = vr.y * s.x - vr.x * s.y - sb.y;
        if (P.distributed) mr += sa * P.w[r];
        Fbus[r] = make_double2(mr, mi);
        if (ip >= 0) {
            x[ip] = (XT)mr;
            lmax = fmax(lmax, fabs(mr));
            lbad |= !isfinite(mr);
        }
        if (iq >= 0) {
            x[iq] = (XT)mi;
            lmax = fmax(lmax, fabs(mi));
            lbad |= !isfinite(mi);
        }
    }
    block_norm(S, lmax, lbad, norm, bad);
}

// dS/dVm and dS/dVa at V scattered into the LU array (and into Jout when requested).
// ZERO_ALL: the LU region (shared memory) is cleared whole with 16-byte stores before the
// entries are written, in place of the gather of the fill-in positions.
template <typename LT, bool ZERO_ALL>
__device__ void jacobian_fill(const DevPlan &P, Shared &S, const double2 *__restrict__ V,
                              const double2 *__restrict__ Ibus, LT *lu, double *Jout) {
    if constexpr (ZERO_ALL) {
        // lu is 4-byte aligned; the head up to the first 16-byte boundary and the tail are scalar
        const int head = (int)(((16 - ((size_t)lu & 15)) & 15) / sizeof(LT));
        const int h = head < P.nnzLU ? head : P.nnzLU;
        if ((int)threadIdx.x < h) lu[threadIdx.x] = (LT)0;
        const int nvec = (P.nnzLU - h) * (int)sizeof(LT) / 16;
        float4 *v4 = reinterpret_cast<float4 *>(lu + h);
        for (int i = threadIdx.x; i < nvec; i += blockDim.x) v4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        const int t0 = h + nvec * 16 / (int)sizeof(LT);
        if ((int)threadIdx.x < P.nnzLU - t0) lu[t0 + threadIdx.x] = (LT)0;
        __syncthreads();
    }
    constexpr int U = 2;  // entries per thread whose loads are issued together
    const int bd = blockDim.x;
    for (int p0 = threadIdx.x; p0 < P.nnzY; p0 += U * bd) {
        int r[U], c[U];
        double2 y[U], vr[U], vc[U], ib[U];
        int4 t[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int p = p0 + u * bd;
            const bool ok = p < P.nnzY;
            r[u] = ok ? P.Rrow[p] : 0;
            c[u] = ok ? P.Rj[p] : 1;
            t[u] = ok ? P.ytarget[p] : make_int4(-1, -1, -1, -1);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int p = p0 + u * bd;
            const bool ok = p < P.nnzY;
            y[u] = ok ? ybus_value(P, S, p) : make_double2(0.0, 0.0);
            vr[u] = ok ? V[r[u]] : make_double2(1.0, 0.0);
            vc[u] = ok ? V[c[u]] : make_double2(1.0, 0.0);
            ib[u] = (ok && r[u] == c[u]) ? Ibus[r[u]] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int p = p0 + u * bd;
            if (p >= P.nnzY) break;
            double dvar, dvai;
            double2 dvm;
            dsbus(y[u], vr[u], vc[u], r[u] == c[u], ib[u], dvar, dvai, dvm);
            if (t[u].x >= 0) lu[t[u].x] = (LT)dvar;
            if (t[u].y >= 0) lu[t[u].y] = (LT)dvai;
            if (t[u].z >= 0) lu[t[u].z] = (LT)dvm.x;
            if (t[u].w >= 0) lu[t[u].w] = (LT)dvm.y;
            if (Jout) {
                const int4 j = P.yjpos[p];
                if (j.x >= 0) Jout[j.x] = dvar;
                if (j.y >= 0) Jout[j.y] = dvai;
                if (j.z >= 0) Jout[j.z] = dvm.x;
                if (j.w >= 0) Jout[j.w] = dvm.y;
            }
        }
    }
    if constexpr (!ZERO_ALL)
        for (int i = threadIdx.x; i < P.nfill; i += blockDim.x) lu[P.fillpos[i]] = (LT)0;
    for (int i = threadIdx.x; i < P.nconst; i += blockDim.x) {
        lu[P.cpos[i]] = (LT)P.cval[i];
        if (Jout) Jout[P.cjpos[i]] = P.cval[i];
    }
}



template <typename LT, typename XT>
__device__ __forceinline__ void run_op(const int4 o, LT *lu, XT *v) {
    const unsigned kind = (unsigned)o.w >> 28;
    const int w = o.w & 0x0fffffff;
    if (kind == 0u) {
        lu[o.x] -= lu[o.y] * lu_div(lu[o.z], lu[w]);
    } else if (kind == 2u) {
        v[o.x] -= lu_div((XT)lu[o.y] * v[o.z], (XT)lu[w]);
    }
    // kind 7: empty slot
}

// Packed operation of the shared-memory layout: s[x] -= s[y] * s[z] / s[w] over the one
// index space of the solve vector and the LU (empty slots write a scratch element).
template <typename T>
__device__ __forceinline__ void run_op_packed(const uint2 o, T *s) {
    const T y = s[o.x >> 16], z = s[o.y & 0xffffu], w = s[o.y >> 16];
    T *px = s + (o.x & 0xffffu);
    *px -= y * lu_div(z, w);
}

struct Trace {
    unsigned long long *buf;
    int cap, n;
    __device__ __forceinline__ void mark() {
        if (buf != nullptr && threadIdx.x == 0 && n < cap) buf[n++] = clock64();
    }
};

// Runs a phase program: one barrier per phase.  In phase p, thread t < sw[p] runs the
// operations sb[p] + t, sb[p] + t + sw[p], ... (bounds and widths staged in shared memory).
//
// Latency hiding: a block barrier also waits for the thread's global loads still in flight,
// so operation loads are not carried across more than the next barrier.  A thread loads the
// first two operations of phase p + 1 when phase p starts (they arrive while phase p works),
// and inside a phase it keeps four operations in flight.  The two register pairs swap roles
// from phase to phase through a loop unrolled by two (a register still waiting for its load
// is never copied).
template <typename OP>
struct OpPair {
    OP a, b;
};

template <typename OP>
__device__ __forceinline__ OP empty_op();
template <>
__device__ __forceinline__ int4 empty_op<int4>() { return make_int4(0, 0, 0, 7 << 28); }

template <typename OP>
__device__ __forceinline__ void load_first2(const OP *__restrict__ ops, const int *sb, const int *sw, int nph,
                                            int p, OpPair<OP> &r, OP none) {
    r.a = none;
    r.b = none;
    if (p < nph) {
        const int w = sw[p];
        if ((int)threadIdx.x < w) {
            const int k = sb[p] + threadIdx.x, e = sb[p + 1];
            if (k < e) r.a = ops[k];
            if (k + w < e) r.b = ops[k + w];
        }
    }
}

template <typename OP, typename F>
__device__ __forceinline__ void run_phase(const OP *__restrict__ ops, const int *sb, const int *sw, int nph, int p,
                                          OpPair<OP> &cur, OpPair<OP> &nxt, OP none, F &&apply, Trace &tr) {
    load_first2<OP>(ops, sb, sw, nph, p + 1, nxt, none);
    const int w = sw[p];
    if ((int)threadIdx.x < w) {
        const int e = sb[p + 1];
        int k = sb[p] + threadIdx.x;
        OP c = none, d = none;
        if (k + 2 * w < e) c = ops[k + 2 * w];
        if (k + 3 * w < e) d = ops[k + 3 * w];
        for (;;) {
            if (k >= e) break;
            apply(cur.a);
            if (k + 4 * w < e) cur.a = ops[k + 4 * w];
            k += w;
            if (k >= e) break;
            apply(cur.b);
            if (k + 4 * w < e) cur.b = ops[k + 4 * w];
            k += w;
            if (k >= e) break;
            apply(c);
            if (k + 4 * w < e) c = ops[k + 4 * w];
            k += w;
            if (k >= e) break;
            apply(d);
            if (k + 4 * w < e) d = ops[k + 4 * w];
            k += w;
        }
    }
    __syncthreads();
    tr.mark();
}

// Phases [a, b) of a program on the first `nwarps` warps: operations from the shared-memory copy
// `sops` (the program's operations from phase a on), one barrier of those warps per phase (no
// global load in flight at it), the other warps go straight to the closing block barrier.
template <typename OP, typename F>
__device__ __forceinline__ void run_narrow(const OP *sops, const int *sb, const int *sw, int a, int b, int nwarps,
                                           F &&apply, Trace &tr) {
    const int nt = nwarps * 32;
    if ((int)threadIdx.x < nt) {
        const int o0 = sb[a];
        for (int p = a; p < b; ++p) {
            const int w = sw[p], e = sb[p + 1] - o0;
            if ((int)threadIdx.x < w)
                for (int k = sb[p] - o0 + threadIdx.x; k < e; k += w) apply(sops[k]);
            asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory");
            tr.mark();
        }
    }
    __syncthreads();
}

template <typename OP, typename F>
__device__ void run_program(const OP *__restrict__ ops, const int *sb, const int *sw, int nph, OP none, F &&apply,
                            Trace &tr) {
    if (nph <= 0) return;
    OpPair<OP> A, B;
    load_first2<OP>(ops, sb, sw, nph, 0, A, none);
    for (int p = 0; p < nph; p += 2) {
        run_phase<OP>(ops, sb, sw, nph, p, A, B, none, apply, tr);
        if (p + 1 >= nph) break;
        run_phase<OP>(ops, sb, sw, nph, p + 1, B, A, none, apply, tr);
    }
}

// The same with phases [na, nb) on the first `nwarps` warps (run_narrow): block-wide phases
// [0, na), the narrow ones, block-wide [nb, nph).
template <typename OP, typename F>
__device__ void run_program_narrow(const OP *__restrict__ ops, const int *sb, const int *sw, int nph, OP none,
                                   F &&apply, Trace &tr, int na, int nb, const OP *sops, int nwarps) {
    if (nph <= 0) return;
    if (nb <= na) na = nb = nph;
    for (int part = 0; part < 2; ++part) {
        const int from = part == 0 ? 0 : nb, to = part == 0 ? na : nph;
        if (from < to) {
            OpPair<OP> A, B;
            load_first2<OP>(ops, sb, sw, to, from, A, none);
            for (int p = from; p < to; p += 2) {
                run_phase<OP>(ops, sb, sw, to, p, A, B, none, apply, tr);
                if (p + 1 >= to) break;
                run_phase<OP>(ops, sb, sw, to, p + 1, B, A, none, apply, tr);
            }
        }
        if (part == 0 && na < nb) run_narrow<OP>(sops, sb, sw, na, nb, nwarps, apply, tr);
    }
}

// One program over the LU layout of the kernel variant: packed operations over the shared
// index space, or int4 operations over the global LU and the shared solve vector.
// NARROW: `nar` is the narrow range of this program (phases [nar.x, nar.y) on nar.z warps,
// operations staged at `sops`), packed layout only.
template <typename LT, typename XT, bool LU_SMEM, bool NARROW = false>
__device__ __forceinline__ void run_lu_program(const uint2 *cops, const int4 *ops, const int *sb, const int *sw,
                                               int nph, int m, LT *lu, XT *x, Trace &tr,
                                               int3 nar = make_int3(0, 0, 0), const uint2 *sops = nullptr) {
    if constexpr (LU_SMEM) {
        static_assert(sizeof(LT) == sizeof(XT), "the packed layout needs one element type");
        const uint2 none = make_uint2((unsigned)m | ((unsigned)m << 16), (unsigned)m | ((unsigned)m << 16));
        if constexpr (NARROW)
            run_program_narrow<uint2>(cops, sb, sw, nph, none, [x](const uint2 o) { run_op_packed<XT>(o, x); }, tr,
                                      nar.x, nar.y, sops, nar.z);
        else
            run_program<uint2>(cops, sb, sw, nph, none, [x](const uint2 o) { run_op_packed<XT>(o, x); }, tr);
    } else {
        run_program<int4>(ops, sb, sw, nph, empty_op<int4>(), [lu, x](const int4 o) { run_op<LT, XT>(o, lu, x); },
                          tr);
    }
}

// z(k) / U(k, k): the backward program keeps z undivided.  CHECK: a zero pivot also sets
// S.piv_err (seen by every thread after the closing barrier).
template <typename LT, typename XT, bool CHECK = false>
__device__ __forceinline__ void scale_by_pivots(const DevPlan &P, Shared &S, const LT *lu, XT *x) {
    int zero = 0;
    for (int k = threadIdx.x; k < P.m; k += blockDim.x) {
        const LT d = lu[P.dpos[k]];
        if (CHECK) zero |= d == (LT)0;
        x[k] = lu_div(x[k], (XT)d);
    }
    if (CHECK && zero) S.piv_err = 1;
    __syncthreads();
}

template <typename LT>
__device__ void check_pivots(const DevPlan &P, Shared &S, const LT *lu) {
    int zero = 0;
    for (int k = threadIdx.x; k < P.m; k += blockDim.x) zero |= lu[P.dpos[k]] == (LT)0;
    if (zero) S.piv_err = 1;
    __syncthreads();
}

// FP64 residual of the Newton system, F - J dx, written as the next right-hand side.  J is the
// linearisation of S(V) = V conj(Y V) in the polar unknowns (the dS/dVa, dS/dVm of
// BaseNRAlgo::_dSbus_dV, BaseNRAlgo.tpp:228-257), so J dx is formed from the voltage
// step dV = V / |V| dVm + j V dVa:  J dx = dV conj(I) + V conj(Y dV)  (I = Y V, the current
// injections of the mismatch), plus the slack-absorption column of a distributed slack.
// Two passes: dV per bus into the slab, then one Ybus row product per equation row.  Returns
// max |F - J dx| to every thread (infinity when a value is not finite).
template <typename XT>
__device__ double newton_residual(const DevPlan &P, Shared &S, const double2 *__restrict__ V,
                                const double2 *__restrict__ Ibus, const double2 *__restrict__ Fbus,
                                const double *__restrict__ dxg, double2 *__restrict__ dV, XT *x) {
    const int bd = blockDim.x;
    for (int b0 = threadIdx.x; b0 < P.n; b0 += 2 * bd) {
        int ia[2], im[2];
        double2 v[2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int b = b0 + i * bd;
            const bool ok = b < P.n;
            ia[i] = ok ? P.xVa[b] : -1;
            im[i] = ok ? P.xVm[b] : -1;
            v[i] = ok ? V[b] : make_double2(1.0, 0.0);
        }
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int b = b0 + i * bd;
            if (b >= P.n) break;
            const double dA = ia[i] >= 0 ? dxg[ia[i]] : 0.0;
            const double dM = im[i] >= 0 ? dxg[im[i]] / cabs2(v[i]) : 0.0;
            dV[b] = make_double2(v[i].x * dM - v[i].y * dA, v[i].y * dM + v[i].x * dA);  // V (dM/|V| + j dA)
        }
    }
    __syncthreads();
    double lmax = 0.0;
    int lbad = 0;
    for (int r = threadIdx.x; r < P.n; r += bd) {
        const int ip = P.xP[r], iq = P.xQ[r];
        if (ip < 0 && iq < 0) continue;
        const double2 yd = ybus_row_product(P, S, dV, r);
        const double2 vr = V[r], dvr = dV[r], ir = Ibus[r];
        double jP = dvr.x * ir.x + dvr.y * ir.y + (vr.x * yd.x + vr.y * yd.y);
        const double jQ = dvr.y * ir.x - dvr.x * ir.y + (vr.y * yd.x - vr.x * yd.y);
        if (P.distributed && ip >= 0) jP += P.wJ[r] * dxg[P.xSlack];
        const double2 F = Fbus[r];
        if (ip >= 0) {
            const double rp = F.x - jP;
            x[ip] = (XT)rp;
            lmax = fmax(lmax, fabs(rp));
            lbad |= !isfinite(rp);
        }
        if (iq >= 0) {
            const double rq = F.y - jQ;
            x[iq] = (XT)rq;
            lmax = fmax(lmax, fabs(rq));
            lbad |= !isfinite(rq);
        }
    }
    double rmax;
    int bad;
    block_norm(S, lmax, lbad, rmax, bad);
    return bad ? INFINITY : rmax;
}
// The voltage update of a Newton step: Va -= dVa, Vm -= dVm (the FP32 step x; when refined, the
// FP64 first step dxg plus xw times the correction x, xw = 0 when the correction was skipped),
// V = Vm e^(j Va) into the slab (and the shared copy Vs); returns the thread's smallest new
// magnitude.  Pairs of buses: their loads (magnitudes and angles, step positions, then
// the step values) are issued together before the arithmetic of the first bus.
// The reference re-derives Vm = |V| and Va = arg(V) before every update (BaseNRSingleSlackAlgo.tpp:
// 131-132), which changes them only where the last magnitude was negative or the angle left
// (-pi, pi]; elsewhere they equal the updated values up to rounding.  So a bus keeps its updated Vm
// and Va and only those buses take |V| and arg(V): two FP64 library calls (and their dependent
// chains) per bus fewer.  The distributed-slack form keeps its own block-wide re-derivation.
template <typename XT>
__device__ double voltage_update(const DevPlan &P, double2 *__restrict__ V, double2 *__restrict__ Vs,
                                           double *__restrict__ Vm, double *__restrict__ Va,
                                           const double *__restrict__ dxg, const XT *x, bool refine_now,
                                           double xw) {
    const int n = P.n;
    double lmin = 1.0;
    constexpr int R = 2;
    const int bd = blockDim.x;
    for (int b0 = threadIdx.x; b0 < n; b0 += R * bd) {
        double vm[R], va[R];
        int ia[R], im[R];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int b = b0 + i * bd;
            const bool ok = b < n;
            ia[i] = ok ? P.xVa[b] : -1;
            im[i] = ok ? P.xVm[b] : -1;
            vm[i] = ok ? Vm[b] : 1.0;
            va[i] = ok ? Va[b] : 0.0;
        }
        double da[R], dm[R];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            da[i] = ia[i] >= 0 ? (refine_now ? dxg[ia[i]] + xw * (double)x[ia[i]] : (double)x[ia[i]]) : 0.0;
            dm[i] = im[i] >= 0 ? (refine_now ? dxg[im[i]] + xw * (double)x[im[i]] : (double)x[im[i]]) : 0.0;
        }
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int b = b0 + i * bd;
            if (b >= n) break;
            double a = va[i], mg = vm[i];
            if (ia[i] >= 0) a -= da[i];
            if (im[i] >= 0) mg -= dm[i];
            double sn, cs;
            sincos(a, &sn, &cs);
            const double2 v = make_double2(mg * cs, mg * sn);
            V[b] = v;
            if (Vs) Vs[b] = v;
            lmin = fmin(lmin, mg);
            if (!P.distributed && !(mg >= 0.0 && fabs(a) <= kPi)) {
                // the reference's re-derivation, where it changes the values (or they are not finite)
                mg = cabs2(v);
                a = atan2(v.y, v.x);
            }
            Vm[b] = mg;
            Va[b] = a;
        }
    }
    return lmin;
}


// ---------------------------------------------------------------- dense tail
// The trailing block of steps [tail_ct, tail_ct + k) of a plan with a dense tail, as a dense
// row-major k x k matrix D in the CTA's slab (row stride tail_ld(k), a multiple of 4 values, so
// that every row starts on 16 bytes).  After the factor program has applied the pivots before
// the block (their updates of the block are the Schur complement of the sparse part),
// tail_factor gathers the block from the LU and factorises it without pivoting, right-looking
// in panels of tail_panel<LT>() columns: (a) the panel (rows [J, k)) staged in shared memory and
// factorised there, one barrier per pivot; then, chunk after chunk of kTailChunk columns right of
// the panel, (b) their U rows staged in shared memory (row stride kTailChunkLd) and solved there,
// a warp per column and a lane per row, the pivots' values passed by shuffles (L of the panel's
// diagonal block is unit lower) and (c) the trailing rows minus L U, each thread a register tile
// of outputs read and written with 16-byte accesses.  Its pivots go back to the LU diagonal,
// where the pivot scaling and the zero-pivot check read them.  Shared memory:
// tail_smem_bytes(k) (the staging area also serves the substitutions' diagonal blocks).
constexpr int kTailChunk = 128;
// row stride of the staged U rows: rows start on 16 bytes, and the lanes of a warp reading one
// column (a lane per row) fall in 8 different banks
constexpr int kTailChunkLd = kTailChunk + 4;
template <typename LT>
__host__ __device__ constexpr int tail_panel() { return sizeof(LT) == 4 ? 32 : 16; }
__host__ __device__ inline int tail_ld(int k) { return (k + 3) & ~3; }
__host__ __device__ inline size_t tail_smem_bytes(int k, int lu_bytes) {
    const int nb = lu_bytes == 4 ? 32 : 16;
    // the panel (k rows of nb + 1 values), then the chunk of U rows from a 16-byte boundary
    return k > 0 ? ((((size_t)k * (nb + 1) + 3) & ~(size_t)3) + (size_t)nb * kTailChunkLd) * lu_bytes : 0;
}

// four consecutive values at a 16-byte boundary
__device__ __forceinline__ void ld4(const float *p, float (&v)[4]) {
    const float4 t = *reinterpret_cast<const float4 *>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void ld4(const double *p, double (&v)[4]) {
    const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void st4(float *p, const float (&v)[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double *p, const double (&v)[4]) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}

template <typename LT>
__device__ __noinline__ void tail_factor(const DevPlan &P, LT *lu, LT *D, LT *sm) {
    constexpr int NB = tail_panel<LT>();
    constexpr int NP = NB + 1;  // panel row stride: the rows of one column fall in different banks
    constexpr int TR = sizeof(LT) == 4 ? 4 : 2, TC = 4;  // register tile of the trailing update
    const int k = P.tail_k, ld = tail_ld(k), tid = threadIdx.x, bd = blockDim.x;
    const int kk = k * k;
    // gather, four entries per thread in flight
    for (int e0 = tid; e0 < kk; e0 += 4 * bd) {
        int p[4];
        LT v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) p[u] = e0 + u * bd < kk ? P.tail_map[e0 + u * bd] : -1;
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = p[u] >= 0 ? lu[p[u]] : (LT)0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = e0 + u * bd;
            if (e < kk) D[(size_t)(e / k) * ld + e % k] = v[u];
        }
    }
    __syncthreads();
    LT *Ap = sm;                     // panel: Ap[(i - J) * NP + c], rows [J, k)
    // U rows of the panel, one chunk: Bc[c * kTailChunkLd + q], from a 16-byte boundary (read with
    // 16-byte loads; sm itself is 16-byte aligned)
    LT *Bc = sm + (((size_t)k * NP + 3) & ~(size_t)3);
    for (int J = 0; J < k; J += NB) {
        const int jb = min(NB, k - J), J1 = J + jb, rows = k - J;
        for (int e = tid; e < rows * NB; e += bd) {
            const int i = e / NB, c = e - i * NB;
            Ap[i * NP + c] = c < jb ? D[(size_t)(J + i) * ld + J + c] : (LT)0;
        }
        __syncthreads();
        // (a) the panel, pivot after pivot
        for (int c = 0; c < jb; ++c) {
            const LT piv = Ap[c * NP + c];
            for (int i = c + 1 + tid; i < rows; i += bd) {
                LT *row = Ap + (size_t)i * NP;
                const LT l = row[c] / piv;
                row[c] = l;
                for (int j = c + 1; j < jb; ++j) row[j] -= l * Ap[c * NP + j];
            }
            __syncthreads();
        }
        for (int e = tid; e < rows * NB; e += bd) {
            const int i = e / NB, c = e - i * NB;
            if (c < jb) D[(size_t)(J + i) * ld + J + c] = Ap[i * NP + c];
        }
        if (J1 >= k) break;
        const int M = k - J1, tr = (M + TR - 1) / TR;
        for (int j0 = J1; j0 < k; j0 += kTailChunk) {
            const int w = min(kTailChunk, k - j0), tc = (w + TC - 1) / TC;
            for (int e = tid; e < NB * kTailChunk; e += bd) {
                const int c = e / kTailChunk, q = e - c * kTailChunk;
                Bc[c * kTailChunkLd + q] = (c < jb && q < w) ? D[(size_t)(J + c) * ld + j0 + q] : (LT)0;
            }
            __syncthreads();
            // (b) the chunk's U rows: a warp per column, lane i holds row i; at step c the lanes
            // below c take row c's final value by a shuffle (the same updates in the same order
            // as a sequential column solve)
            {
                const int lane = tid & 31, nwarps = bd >> 5;
                for (int q = tid >> 5; q < w; q += nwarps) {
                    LT v = lane < jb ? Bc[lane * kTailChunkLd + q] : (LT)0;
                    for (int c = 0; c + 1 < jb; ++c) {
                        const LT u = __shfl_sync(0xffffffffu, v, c);
                        if (lane > c && lane < jb) v -= Ap[lane * NP + c] * u;
                    }
                    if (lane < jb) Bc[lane * kTailChunkLd + q] = v;
                }
            }
            __syncthreads();
            for (int e = tid; e < jb * kTailChunk; e += bd) {
                const int c = e / kTailChunk, q = e - c * kTailChunk;
                if (q < w) D[(size_t)(J + c) * ld + j0 + q] = Bc[c * kTailChunkLd + q];
            }
            // (c) the trailing rows: a tile of TR rows x 4 columns per thread (columns past the
            // block's last fall in the row padding; their values are never read as entries)
            for (int t = tid; t < tr * tc; t += bd) {
                const int ti = t / tc, tj = t - ti * tc;
                const int i0 = J1 + ti * TR, q0 = tj * TC;
                LT acc[TR][TC];
#pragma unroll
                for (int r = 0; r < TR; ++r) {
                    if (i0 + r < k) ld4(D + (size_t)(i0 + r) * ld + j0 + q0, acc[r]);
                    else acc[r][0] = acc[r][1] = acc[r][2] = acc[r][3] = (LT)0;
                }
                const LT *arow = Ap + (size_t)(i0 - J) * NP;
#pragma unroll 4
                for (int c = 0; c < NB; ++c) {
                    LT a[TR], bq[TC];
#pragma unroll
                    for (int r = 0; r < TR; ++r) a[r] = i0 + r < k ? arow[r * NP + c] : (LT)0;
                    ld4(Bc + c * kTailChunkLd + q0, bq);
#pragma unroll
                    for (int r = 0; r < TR; ++r)
#pragma unroll
                        for (int q = 0; q < TC; ++q) acc[r][q] -= a[r] * bq[q];
                }
#pragma unroll
                for (int r = 0; r < TR; ++r)
                    if (i0 + r < k) st4(D + (size_t)(i0 + r) * ld + j0 + q0, acc[r]);
            }
            __syncthreads();
        }
    }
    __syncthreads();
    for (int c = tid; c < k; c += bd) lu[P.dpos[P.tail_ct + c]] = D[(size_t)c * ld + c];
    __syncthreads();
}

// Forward substitution of the block (unit lower L of tail_factor) on x[tail_ct, tail_ct + k),
// after the forward pushes of the pivots before the block: per panel of 32 rows, the diagonal
// block staged in shared memory (`sm`, row stride 33), warp 0 solves it (a lane per row, values exchanged by
// shuffles), then every thread updates rows below it.
template <typename LT, typename XT>
__device__ __noinline__ void tail_forward(const DevPlan &P, const LT *D, XT *x, LT *sm) {
    const int k = P.tail_k, ld = tail_ld(k), tid = threadIdx.x, bd = blockDim.x;
    XT *xt = x + P.tail_ct;
    for (int J = 0; J < k; J += 32) {
        const int jb = min(32, k - J), J1 = J + jb;
        for (int e = tid; e < jb * 32; e += bd) {
            const int a = e >> 5, b = e & 31;
            sm[a * 33 + b] = b < jb ? D[(size_t)(J + a) * ld + J + b] : (LT)0;
        }
        __syncthreads();
        if (tid < 32) {
            XT v = tid < jb ? xt[J + tid] : (XT)0;
            for (int c = 0; c < jb; ++c) {
                const XT vc = __shfl_sync(0xffffffffu, v, c);
                if (tid > c && tid < jb) v -= (XT)sm[tid * 33 + c] * vc;
            }
            if (tid < jb) xt[J + tid] = v;
        }
        __syncthreads();
        for (int i = J1 + tid; i < k; i += bd) {
            XT v = xt[i];
            const LT *row = D + (size_t)i * ld + J;
            for (int c = 0; c < jb; ++c) v -= (XT)row[c] * xt[J + c];
            xt[i] = v;
        }
        __syncthreads();
    }
}

// Backward substitution of the block, before the backward program, in its convention: the values
// stay undivided (z(c) = U(c, c) x(c)) and a push divides by the pivot; the pivot scaling after
// the program divides them.  Per panel from the last: the diagonal block staged in shared
// memory, warp 0 solves it and leaves the panel's z(c) / U(c, c) in S.red, then every thread
// updates the rows above it.
template <typename LT, typename XT>
__device__ __noinline__ void tail_backward(const DevPlan &P, Shared &S, const LT *D, XT *x, LT *sm) {
    const int k = P.tail_k, ld = tail_ld(k), tid = threadIdx.x, bd = blockDim.x;
    XT *xt = x + P.tail_ct;
    const int last = ((k - 1) / 32) * 32;
    for (int J = last; J >= 0; J -= 32) {
        const int jb = min(32, k - J);
        for (int e = tid; e < jb * 32; e += bd) {
            const int a = e >> 5, b = e & 31;
            sm[a * 33 + b] = b < jb ? D[(size_t)(J + a) * ld + J + b] : (LT)0;
        }
        __syncthreads();
        if (tid < 32) {
            XT z = tid < jb ? xt[J + tid] : (XT)0;
            for (int c = jb - 1; c >= 0; --c) {
                const XT zc = __shfl_sync(0xffffffffu, z, c);
                const XT w = zc / (XT)sm[c * 33 + c];
                if (tid == c) S.red[c] = (double)w;
                if (tid < c) z -= (XT)sm[tid * 33 + c] * w;
            }
            if (tid < jb) xt[J + tid] = z;
        }
        __syncthreads();
        for (int i = tid; i < J; i += bd) {
            XT v = xt[i];
            const LT *row = D + (size_t)i * ld + J;
            for (int c = 0; c < jb; ++c) v -= (XT)row[c] * (XT)S.red[c];
            xt[i] = v;
        }
        __syncthreads();
    }
}

// Where one plan's data lives for a CTA: shared memory x | LU (LU_SMEM: one index space, LU at
// element lu_offset) | phase tables, and the CTA's slab of the scratch memory.
// slab bytes per bus: V, Ibus, Fbus, the refinement's voltage step dV (16 B each), Vm, Va (8 B each)
constexpr size_t kBusSlabBytes = 80;
template <typename LT, typename XT>
struct Layout {
    XT *x;
    LT *lu;
    LT *D;    // dense tail block (global-memory LU plans with a tail)
    LT *tsm;  // its staging area in shared memory
    double2 *V, *Ibus, *Fbus, *dV;
    double *Vm, *Va, *dxg;
    int *sb_fac, *sb_bwd, *sb_fwd, *sw_fac, *sw_bwd, *sw_fwd;
    uint2 *nar_ops[3];  // staged operations of the narrow phases (packed layout)
};

template <typename LT, typename XT, bool LU_SMEM>
__device__ __forceinline__ Layout<LT, XT> make_layout(const DevPlan &P, const BatchArgs &A, unsigned char *dyn) {
    Layout<LT, XT> L;
    const int n = P.n, m = P.m;
    const size_t xbytes = LU_SMEM ? (size_t)P.lu_offset * sizeof(XT) : (((size_t)m * sizeof(XT) + 15) & ~(size_t)15);
    L.x = reinterpret_cast<XT *>(dyn);
    unsigned char *slab = A.scratch + (size_t)blockIdx.x * (size_t)A.slab_bytes;
    L.V = reinterpret_cast<double2 *>(slab);
    L.Ibus = L.V + n;
    L.Fbus = L.Ibus + n;
    L.dV = L.Fbus + n;
    L.Vm = reinterpret_cast<double *>(L.dV + n);
    L.Va = L.Vm + n;
    L.dxg = L.Va + n;
    const size_t bus_bytes = (((size_t)n * kBusSlabBytes + (size_t)m * 8) + 255) & ~(size_t)255;
    L.lu = LU_SMEM ? reinterpret_cast<LT *>(dyn + xbytes) : reinterpret_cast<LT *>(slab + bus_bytes);
    L.D = LU_SMEM ? nullptr
                  : reinterpret_cast<LT *>(slab + bus_bytes + (((size_t)P.nnzLU * sizeof(LT) + 255) & ~(size_t)255));
    L.sb_fac = reinterpret_cast<int *>(dyn + xbytes +
                                       (LU_SMEM ? (((size_t)P.nnzLU * sizeof(LT) + 15) & ~(size_t)15) : 0));
    L.sb_bwd = L.sb_fac + P.fac_nph + 1;
    L.sb_fwd = L.sb_bwd + P.bwd_nph + 1;
    L.sw_fac = L.sb_fwd + P.fwd_nph + 1;
    L.sw_bwd = L.sw_fac + P.fac_nph;
    L.sw_fwd = L.sw_bwd + P.bwd_nph;
    {
        // the narrow phases' operations after the tables, 8-byte aligned
        const size_t off = (size_t)((reinterpret_cast<unsigned char *>(L.sw_fwd + P.fwd_nph) - dyn + 7) & ~(size_t)7);
        uint2 *base = reinterpret_cast<uint2 *>(dyn + off);
        for (int k = 0; k < 3; ++k) L.nar_ops[k] = base + P.nar_off[k];
        // the dense tail's staging area after the tables, 16-byte aligned (global-memory LU)
        L.tsm = LU_SMEM ? nullptr : reinterpret_cast<LT *>(dyn + ((off + 15) & ~(size_t)15));
    }
    return L;
}

// Phase bounds and widths of the three programs into shared memory (caller synchronises).
template <typename LT, typename XT>
__device__ __forceinline__ void stage_tables(const DevPlan &P, const Layout<LT, XT> &L) {
    for (int i = threadIdx.x; i <= P.fac_nph; i += blockDim.x) L.sb_fac[i] = P.fac_base[i];
    for (int i = threadIdx.x; i <= P.bwd_nph; i += blockDim.x) L.sb_bwd[i] = P.bwd_base[i];
    for (int i = threadIdx.x; i <= P.fwd_nph; i += blockDim.x) L.sb_fwd[i] = P.fwd_base[i];
    for (int i = threadIdx.x; i < P.fac_nph; i += blockDim.x) L.sw_fac[i] = P.fac_width[i];
    for (int i = threadIdx.x; i < P.bwd_nph; i += blockDim.x) L.sw_bwd[i] = P.bwd_width[i];
    for (int i = threadIdx.x; i < P.fwd_nph; i += blockDim.x) L.sw_fwd[i] = P.fwd_width[i];
    if (P.compact) {
        const uint2 *cops[3] = {P.fac_cops, P.bwd_cops, P.fwd_cops};
        for (int k = 0; k < 3; ++k) {
            const int cnt = P.nar_off[k + 1] - P.nar_off[k];
            for (int i = threadIdx.x; i < cnt; i += blockDim.x) L.nar_ops[k][i] = cops[k][P.nar_first[k] + i];
        }
    }
}

// Per-phase SM cycles, measured by thread 0 between the barriers that end each phase.
struct Prof {
    bool on;
    int traced;
    unsigned long long tmark;
    unsigned long long *pc;  // Shared::pc: the counters stay out of the registers
    __device__ __forceinline__ void start(bool o, unsigned long long *counters) {
        on = o;
        traced = 0;
        pc = counters;
        tmark = o ? clock64() : 0;
        if (o)
            for (int i = 0; i < kPhaseSlots; ++i) pc[i] = 0;
    }
    __device__ __forceinline__ void mark(int slot) {
        if (on) {
            const unsigned long long t = clock64();
            pc[slot] += t - tmark;
            tmark = t;
        }
    }
};

// One job: instances [first, first + count) of a batch, chained for a time series.  The batch's
// inputs (start voltages, injections, overrides) are read through L2 only (ld.global.cg): in the
// device-resident request loop one launch serves many requests whose inputs reuse device
// addresses, and an SM's L1 could still hold an earlier request's lines.
// NARROW: the narrow phases of the packed programs run on their few warps (the 512- and
// 640-thread variants; at 768 threads the registers it takes cost more than it saves).
template <typename LT, typename XT, bool LU_SMEM, bool REFINE, bool NARROW>
__device__ __forceinline__ void solve_job(const DevPlan &P, const BatchArgs &A, Shared &S, const Layout<LT, XT> &L,
                                          int first, int count, Prof &pr) {
    const int tid = threadIdx.x;
    const int n = P.n, m = P.m;
    XT *x = L.x;
    LT *lu = L.lu;
    double2 *V = L.V, *Ibus = L.Ibus, *Fbus = L.Fbus;
    double *Vm = L.Vm, *Va = L.Va, *dxg = L.dxg;
    // With the LU in shared memory, the LU region is dead from the voltage update to the next
    // Jacobian fill: the voltages are also written there (Vs) and the mismatch gathers them from
    // shared memory instead of the slab.  Not when the LU must survive the mismatch (LU reuse).
    double2 *Vs = nullptr;
    if constexpr (LU_SMEM) {
        if (!(REFINE && A.reuse_below > 0.0) && (size_t)n * sizeof(double2) <= (size_t)P.nnzLU * sizeof(LT))
            Vs = reinterpret_cast<double2 *>(lu);
    }
    for (int step = 0; step < count; ++step) {
        const int inst = first + step;
        const double2 *Sb = A.Sbus + (long long)inst * A.sbus_stride;
        if (step == 0 || !A.chain) {
            const double2 *v0 = A.v0_from_out ? out_row(A, inst, n) : A.V0 + (long long)inst * A.v0_stride;
            for (int b = tid; b < n; b += blockDim.x) {
                const double2 v = __ldcg(v0 + b);
                V[b] = v;
                if (Vs) Vs[b] = v;
                Vm[b] = cabs2(v);
                Va[b] = atan2(v.y, v.x);
            }
        } else {
            for (int b = tid; b < n; b += blockDim.x) {
                const double2 v = V[b];
                if (Vs) Vs[b] = v;
                Vm[b] = cabs2(v);
                Va[b] = atan2(v.y, v.x);
            }
        }
        if (tid == 0) {
            int k0 = 0, k1 = 0;
            if (A.ovr_ptr) {
                k0 = __ldcg(A.ovr_ptr + inst);
                k1 = __ldcg(A.ovr_ptr + inst + 1);
            }
            S.novr = k1 - k0 > kMaxOverrides ? -1 : k1 - k0;  // -1: too many to stage
            S.piv_err = 0;
            S.slack_absorbed = 0.0;
        }
        __syncthreads();
        if (tid < S.novr) {
            const int k0 = __ldcg(A.ovr_ptr + inst);
            S.opos[tid] = __ldcg(A.ovr_pos + k0 + tid);
            S.oval[tid] = __ldcg(A.ovr_val + k0 + tid);
        }
        if (P.distributed) {
            double ls = 0.0;
            for (int b = tid; b < n; b += blockDim.x) ls += __ldcg(Sb + b).x;
            const double tot = block_sum(S, ls);
            if (tid == 0) S.slack_absorbed = tot;
        }
        __syncthreads();
        if (S.novr < 0) {
            // more Ybus overrides than the kernel stages: not computed (start voltages out)
            double2 *vo = out_row(A, inst, n);
            for (int b = tid; b < n; b += blockDim.x) vo[b] = A.zero_failed ? make_double2(0.0, 0.0) : V[b];
            if (tid == 0) {
                A.iters[inst] = 0;
                A.errs[inst] = 8;  // NotInitError
            }
            __syncthreads();
            if (A.chain) {
                for (int s2 = step + 1 + tid; s2 < count; s2 += blockDim.x) {
                    A.iters[first + s2] = 0;
                    A.errs[first + s2] = 8;
                }
                break;
            }
            continue;
        }
        double norm;
        int bad;
        pr.mark(6);
        mismatch<XT>(P, S, Vs ? Vs : V, Ibus, Fbus, Sb, x, norm, bad);
        pr.mark(0);
        bool conv = !bad && norm < A.tol;
        int it = A.it_start ? A.it_start[inst] : 0, err = 0;
        double *Jout = (A.Jout && inst == A.j_inst) ? A.Jout : nullptr;
        Trace tr{(A.trace != nullptr && blockIdx.x == 0 && pr.traced == 0) ? A.trace : nullptr, A.trace_cap, 0};
        pr.traced = 1;
        bool have_lu = false;  // this instance's LU from an earlier iteration is in place
        while (!conv && it < A.max_iter) {
            ++it;
            const bool refine_now = REFINE && norm < A.refine_below;
            // close to the solution the Jacobian barely moves between iterations: the step is
            // solved with the previous iteration's LU and refined against the current FP64
            // Jacobian (refine_now holds: reuse_below <= refine_below)
            const bool reuse = REFINE && have_lu && Jout == nullptr && norm < A.reuse_below;
            tr.mark();
            if (!reuse) {
                jacobian_fill<LT, LU_SMEM>(P, S, V, Ibus, lu, Jout);
                __syncthreads();
                pr.mark(1);
                // refactorisation with the forward substitution of the right-hand side fused in
                run_lu_program<LT, XT, LU_SMEM, NARROW>(P.fac_cops, P.fac_ops, L.sb_fac, L.sw_fac, P.fac_nph, m, lu, x, tr,
                                                make_int3(P.nar_a[0], P.nar_b[0], P.nar_warps), L.nar_ops[0]);
                if constexpr (!LU_SMEM) {
                    if (P.tail_k > 0) {
                        tail_factor<LT>(P, lu, L.D, L.tsm);
                        tail_forward<LT, XT>(P, L.D, x, L.tsm);
                    }
                }
                pr.mark(2);
                have_lu = true;
            } else {
                run_lu_program<LT, XT, LU_SMEM, NARROW>(P.fwd_cops, P.fwd_ops, L.sb_fwd, L.sw_fwd, P.fwd_nph, m, lu, x, tr,
                                                make_int3(P.nar_a[2], P.nar_b[2], P.nar_warps), L.nar_ops[2]);
                if constexpr (!LU_SMEM) {
                    if (P.tail_k > 0) tail_forward<LT, XT>(P, L.D, x, L.tsm);
                }
                pr.mark(3);
            }
            if constexpr (!LU_SMEM) {
                if (P.tail_k > 0) tail_backward<LT, XT>(P, S, L.D, x, L.tsm);
            }
            run_lu_program<LT, XT, LU_SMEM, NARROW>(P.bwd_cops, P.bwd_ops, L.sb_bwd, L.sw_bwd, P.bwd_nph, m, lu, x, tr,
                                            make_int3(P.nar_a[1], P.nar_b[1], P.nar_warps), L.nar_ops[1]);
            // a zero pivot of the refactorisation is detected here: the backward program ran on
            // non-finite values, which are dropped with the step
            scale_by_pivots<LT, XT, true>(P, S, lu, x);
            if (S.piv_err) {
                err = 6;  // SolverReFactor
                break;
            }
            pr.mark(4);
            // the refinement's correction solve is skipped when the residual of the FP32 step is
            // below a hundredth of the tolerance: the correction would move the next mismatch by
            // less than that (J e = r), and the final voltages by at most |J^-1| tol / 100
            double xw = 1.0;
            if (refine_now) {
                for (int k = tid; k < m; k += blockDim.x) dxg[k] = (double)x[k];
                __syncthreads();
                const double rmax = newton_residual<XT>(P, S, V, Ibus, Fbus, dxg, L.dV, x);
                if (rmax < 0.01 * A.tol) xw = 0.0;
            }
            if (refine_now && xw != 0.0) {
                __syncthreads();
                run_lu_program<LT, XT, LU_SMEM, NARROW>(P.fwd_cops, P.fwd_ops, L.sb_fwd, L.sw_fwd, P.fwd_nph, m, lu, x, tr,
                                                make_int3(P.nar_a[2], P.nar_b[2], P.nar_warps), L.nar_ops[2]);
                if constexpr (!LU_SMEM) {
                    if (P.tail_k > 0) {
                        tail_forward<LT, XT>(P, L.D, x, L.tsm);
                        tail_backward<LT, XT>(P, S, L.D, x, L.tsm);
                    }
                }
                run_lu_program<LT, XT, LU_SMEM, NARROW>(P.bwd_cops, P.bwd_ops, L.sb_bwd, L.sw_bwd, P.bwd_nph, m, lu, x, tr,
                                            make_int3(P.nar_a[1], P.nar_b[1], P.nar_warps), L.nar_ops[1]);
                scale_by_pivots<LT, XT>(P, S, lu, x);
            }
            if (refine_now) pr.mark(5);
            // voltage update
            const double lmin = voltage_update<XT>(P, V, Vs, Vm, Va, dxg, x, refine_now, xw);
            if (P.distributed) {
                const double dxs =
                    refine_now ? dxg[P.xSlack] + xw * (double)x[P.xSlack] : (double)x[P.xSlack];
                const double vmin = block_min(S, lmin);  // contains barriers
                if (tid == 0) S.slack_absorbed -= dxs;
                if (vmin < 0.0) {
                    for (int b = tid; b < n; b += blockDim.x) {
                        const double2 v = V[b];
                        Vm[b] = cabs2(v);
                        Va[b] = atan2(v.y, v.x);
                    }
                }
            }
            __syncthreads();
            tr.mark();
            tr.buf = nullptr;
            pr.mark(6);
            mismatch<XT>(P, S, Vs ? Vs : V, Ibus, Fbus, Sb, x, norm, bad);
            pr.mark(0);
            if (bad) {
                err = 3;  // InifiniteValue
                break;
            }
            conv = norm < A.tol;
        }
        if (!conv && err == 0) err = 2;  // TooManyIterations
        double2 *vo = out_row(A, inst, n);
        const bool zero = A.zero_failed && err != 0;
        for (int b = tid; b < n; b += blockDim.x) vo[b] = zero ? make_double2(0.0, 0.0) : V[b];
        if (tid == 0) {
            A.iters[inst] = it;
            A.errs[inst] = err;
            if (pr.on) pr.pc[7] += 1;
        }
        __syncthreads();
        if (A.chain && err != 0) {
            // the reference stops a time series at its first divergence
            for (int s2 = step + 1 + tid; s2 < count; s2 += blockDim.x) {
                A.iters[first + s2] = 0;
                A.errs[first + s2] = 8;  // NotInitError: not computed
            }
            break;
        }
    }
}

// The mixed form's FP64 fallback inside the launch: a job with an instance that did not converge
// in FP32 is solved again in FP64 by the same CTA, with the solve vector in the shared memory
// the FP32 LU used (the next job refills it) and the FP64 LU in the CTA's slab.  The same code
// as a separate FP64 launch (solve_job with FP64 LU in global memory); a function of its own so
// that its registers do not add to the FP32 path's.
__device__ __noinline__ void fp64_rerun(const DevPlan &P, const BatchArgs &A, Shared &S, unsigned char *dyn,
                                        int first, int count) {
    const Layout<double, double> L = make_layout<double, double, false>(P, A, dyn);
    stage_tables<double, double>(P, L);
    __syncthreads();
    Prof pr;
    pr.start(false, S.pc);
    solve_job<double, double, false, false, false>(P, A, S, L, first, count, pr);
}

// QUEUE: the device-resident request loop (jobs from M.q); a variant of its own so that the
// other launches keep their registers.
// MAXT: the launch bound, 512, 640 or 768 threads.  More warps hide more of the phases' latency
// at fewer registers per thread (128, 96, 80): the large plans run 640 (mixed form, with the
// narrow phases on a few warps) or 768 threads (FP64 form).
template <typename LT, typename XT, bool LU_SMEM, bool REFINE, bool QUEUE, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) nr_batch_kernel(const DevPlan P0, const BatchArgs A0, const MultiArgs M) {
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ Shared S;
    // the plan and batch of the current job, in shared memory: a launch of one plan (M.segs
    // null) copies its parameters once; a launch over several plans copies the segment of a
    // job when it differs from the CTA's previous one and restages the phase tables.  Both
    // kinds run the same code, so an instance gives the same bits in either.
    __shared__ __align__(16) Segment seg;
    const int tid = threadIdx.x;
    constexpr bool queue = QUEUE;
    const bool multi = M.segs != nullptr || queue;
    int *const counter = multi ? M.job_counter : A0.job_counter;
    const int njobs = multi ? M.njobs : (A0.njobs_dev ? min(A0.njobs, *A0.njobs_dev) : A0.njobs);
    Prof pr;
    pr.start(A0.phase_cycles != nullptr && tid == 0, S.pc);
    int cur = -1;
    Layout<LT, XT> L{};
    __shared__ QueueJob qjob;
    for (;;) {
        if constexpr (QUEUE) {
            // request loop: claim the next published job (compare-and-swap on the head, so a CTA
            // never holds a job that is not there yet); after idle_polls empty polls, leave
            if (tid == 0)
                S.job = claim_queue_job(M.q.jobs, M.q.cap, M.q.head, M.q.tail, M.q.closing, M.q.idle_polls, &qjob);
            __syncthreads();
            const int got = S.job;
            __syncthreads();
            if (got < 0) break;
        } else {
            if (tid == 0) S.job = atomicAdd(counter, 1);
            __syncthreads();
            const int job = S.job;
            __syncthreads();
            if (job >= njobs) break;
        }
        const int job = S.job;
        // a request loop keys the segment a CTA holds by the request's sequence number (slots
        // are reused by later requests)
        const int sj = queue ? qjob.req : (multi ? M.job_seg[job] : 0);
        if (sj != cur) {
            if (multi) {
                static_assert(sizeof(Segment) % sizeof(int4) == 0, "segment records are copied as int4");
                const int4 *src = reinterpret_cast<const int4 *>(queue ? M.q.segs + qjob.slot : M.segs + sj);
                int4 *dst = reinterpret_cast<int4 *>(&seg);
                for (int i = tid; i < (int)(sizeof(Segment) / sizeof(int4)); i += blockDim.x) dst[i] = __ldcg(src + i);
            } else if (tid == 0) {
                seg.P = P0;
                seg.A = A0;
            }
            __syncthreads();
            cur = sj;
            L = make_layout<LT, XT, LU_SMEM>(seg.P, seg.A, dyn);
            stage_tables<LT, XT>(seg.P, L);
            __syncthreads();
        }
        const int first = queue ? qjob.first : (multi ? M.job_first[job] : A0.job_first[job]);
        const int count = queue ? qjob.count : (multi ? M.job_count[job] : A0.job_count[job]);
        solve_job<LT, XT, LU_SMEM, REFINE, (MAXT <= 640)>(seg.P, seg.A, S, L, first, count, pr);
        __syncthreads();
        if constexpr (REFINE) {
            if (seg.A.fp64_inline) {
                if (tid == 0) {
                    int bad = 0;
                    for (int i = first; i < first + count; ++i) bad |= seg.A.errs[i] != 0;
                    S.job_failed = bad;
                }
                __syncthreads();
                if (S.job_failed) {
                    // the word after the job counter counts the instances re-solved in FP64; the
                    // re-solve starts afresh from the instance's start voltages
                    const int *its = seg.A.it_start;
                    const int vfo = seg.A.v0_from_out;
                    if (tid == 0) {
                        if (seg.A.job_counter != nullptr) atomicAdd(seg.A.job_counter + 1, count);
                        seg.A.it_start = nullptr;
                        seg.A.v0_from_out = 0;
                    }
                    __syncthreads();
                    fp64_rerun(seg.P, seg.A, S, dyn, first, count);
                    __syncthreads();
                    if (tid == 0) {
                        seg.A.it_start = its;
                        seg.A.v0_from_out = vfo;
                    }
                    stage_tables<LT, XT>(seg.P, L);  // the FP64 solve vector covered them
                    __syncthreads();
                }
            }
        }
        if constexpr (QUEUE) {
            if (tid == 0) signal_queue_job(M.q.done, qjob.slot, count);
        }
    }
    if (pr.on)
        for (int i = 0; i < kPhaseSlots; ++i) A0.phase_cycles[(size_t)blockIdx.x * kPhaseSlots + i] = pr.pc[i];
}

}  // namespace

// Raises a kernel's dynamic shared-memory limit to everything the device allows, once per
// kernel and device (launches then pass their own size; setting the attribute on every
// launch would make concurrent launches on other streams wait on the driver).
cudaError_t allow_max_smem(const void *fn) {
    static std::mutex mu;
    static std::set<std::pair<const void *, int>> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (done.count({fn, dev})) return cudaSuccess;
    int optin = 0;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    if (e != cudaSuccess) return e;
    done.insert({fn, dev});
    return cudaSuccess;
}

namespace {

// DC power flow of a batch (BaseDCAlgo::compute_pf, src/powerflow_algorithm/BaseDCAlgo.tpp:
// 86-175), FP64, one CTA per instance: B from the real parts of the instance's Ybus (overrides
// applied), right-hand side Re(Sbus) at the non-slack buses, refactorisation with the forward
// substitution fused, backward substitution; the angles are shifted by the slack's start angle,
// the magnitudes are the start magnitudes.  A non-finite solution or one with |theta| >= 1e6 is
// SolverSolve (:115-123): zero voltages.  One linear solve: iters = 1.
template <bool LU_SMEM>
__global__ void __launch_bounds__(512, 1) dc_batch_kernel(const DevPlan P, const BatchArgs A) {
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ Shared S;
    const int tid = threadIdx.x;
    const int n = P.n, m = P.m;
    const Layout<double, double> L = make_layout<double, double, LU_SMEM>(P, A, dyn);
    stage_tables<double, double>(P, L);
    __syncthreads();
    double *x = L.x, *lu = L.lu;
    Trace tr{nullptr, 0, 0};
    for (;;) {
        if (tid == 0) S.job = atomicAdd(A.job_counter, 1);
        __syncthreads();
        const int job = S.job;
        __syncthreads();
        if (job >= A.njobs) break;
        const int first = A.job_first[job], count = A.job_count[job];
        for (int inst = first; inst < first + count; ++inst) {
            if (tid == 0) {
                int k0 = 0, k1 = 0;
                if (A.ovr_ptr) {
                    k0 = A.ovr_ptr[inst];
                    k1 = A.ovr_ptr[inst + 1];
                }
                S.novr = k1 - k0 > kMaxOverrides ? -1 : k1 - k0;  // -1: too many to stage
                S.piv_err = 0;
            }
            __syncthreads();
            if (tid < S.novr) {
                const int k0 = A.ovr_ptr[inst];
                S.opos[tid] = A.ovr_pos[k0 + tid];
                S.oval[tid] = A.ovr_val[k0 + tid];
            }
            __syncthreads();
            if (S.novr < 0) {
                // more Ybus overrides than the kernel stages: not computed (start voltages out)
                const double2 *v0 = A.V0 + (long long)inst * A.v0_stride;
                double2 *vo = out_row(A, inst, n);
                for (int b = tid; b < n; b += blockDim.x) vo[b] = A.zero_failed ? make_double2(0.0, 0.0) : v0[b];
                if (tid == 0) {
                    A.iters[inst] = 0;
                    A.errs[inst] = 8;  // NotInitError
                }
                __syncthreads();
                continue;
            }
            for (int p = tid; p < P.nnzY; p += blockDim.x) {
                const int t = P.ytarget[p].x;
                if (t >= 0) lu[t] = ybus_value(P, S, p).x;
            }
            for (int i = tid; i < P.nfill; i += blockDim.x) lu[P.fillpos[i]] = 0.0;
            const double2 *Sb = A.Sbus + (long long)inst * A.sbus_stride;
            for (int b = tid; b < n; b += blockDim.x) {
                const int ip = P.xP[b];
                if (ip >= 0) x[ip] = Sb[b].x;
            }
            __syncthreads();
            run_lu_program<double, double, LU_SMEM>(P.fac_cops, P.fac_ops, L.sb_fac, L.sw_fac, P.fac_nph, m, lu, x,
                                                    tr);
            check_pivots<double>(P, S, lu);
            int err = 0;
            if (S.piv_err) {
                err = 6;  // SolverReFactor
            } else {
                run_lu_program<double, double, LU_SMEM>(P.bwd_cops, P.bwd_ops, L.sb_bwd, L.sw_bwd, P.bwd_nph, m, lu,
                                                        x, tr);
                scale_by_pivots<double, double>(P, S, lu, x);
                double lmax = 0.0;
                int lbad = 0;
                for (int k = tid; k < m; k += blockDim.x) {
                    lmax = fmax(lmax, fabs(x[k]));
                    lbad |= !isfinite(x[k]);
                }
                double nrm;
                int bad;
                block_norm(S, lmax, lbad, nrm, bad);
                if (bad || nrm >= 1e6) err = 7;  // SolverSolve
            }
            const double2 *v0 = A.V0 + (long long)inst * A.v0_stride;
            double2 *vo = out_row(A, inst, n);
            const double2 vs = v0[P.slack0];
            const double a0 = atan2(vs.y, vs.x);
            for (int b = tid; b < n; b += blockDim.x) {
                double2 v = make_double2(0.0, 0.0);
                if (err == 0) {
                    const int ia = P.xVa[b];
                    const double va = (ia >= 0 ? x[ia] : 0.0) + a0;
                    const double vm = cabs2(v0[b]);
                    double sn, cs;
                    sincos(va, &sn, &cs);
                    v = make_double2(vm * cs, vm * sn);
                }
                vo[b] = v;
            }
            if (tid == 0) {
                A.iters[inst] = err == 0 ? 1 : 0;
                A.errs[inst] = err;
            }
            __syncthreads();
        }
    }
}

// Fast decoupled power flow of a batch (BaseFDPFAlgo::compute_pf, src/powerflow_algorithm/
// BaseFDPFAlgo.tpp:11-173, with has_converged, BaseFDPFAlgo.hpp:118-170), FP64, one CTA per
// instance.  B' (over pvpq) and B'' (over pq) were factorised when the plan was built and do
// not change between instances (the reference's batch computers keep the base factors for
// every contingency and step); each CTA copies both factors into its shared memory once when
// they fit, else reads them from global memory (one copy, L2 resident).  An iteration:
//   P half-step  dVa = B'^-1 P, Va[pvpq] -= dVa, t = exp(j Va), V = Vm t, (Vm, Va) = (|V|, arg V)
//   Q half-step  dVm = B''^-1 Q, Vm[pq] -= dVm, V = Vm t, (Vm, Va) = (|V|, arg V)
// each followed by the mismatch  mis = (V conj(Ybus V) - Sbus + slack_absorbed w) / Vm,
// P = Re(mis)[pvpq], Q = Im(mis)[pq], converged when max(|P|, |Q|) < tol, InifiniteValue when
// any bus's mis is not finite; slack_absorbed = Re(sum Sbus), the reference's start value,
// which its FDPF never updates.
// Only one of P and Q is needed at a time (P before a B' solve, Q before a B'' solve), so the
// two systems share one solve vector; with the factors in shared memory the index space is
// x | LU(B') | LU(B''), each system's packed operations addressing its LU at its lu_offset.
struct FdpfLayout {
    double *x[2];         // the shared solve vector (both entries equal)
    const double *lu[2];  // factor values (shared or global)
    int *sbf[2], *swf[2], *sbb[2], *swb[2];
    double2 *V, *T;       // voltages, exp(j Va) of the last P half-step
    double *Vm, *Va;
};

__host__ __device__ __forceinline__ size_t fdpf_region_bytes(const DevPlan &B0, const DevPlan &B1, bool lu_in_smem) {
    const size_t e0 = lu_in_smem ? (size_t)B0.lu_offset + (size_t)B0.nnzLU : (size_t)B0.m + 1;
    const size_t e1 = lu_in_smem ? (size_t)B1.lu_offset + (size_t)B1.nnzLU : (size_t)B1.m + 1;
    const size_t e = e0 > e1 ? e0 : e1;
    return (e * sizeof(double) + 15) & ~(size_t)15;
}

// B: the two systems' plans (in shared memory)
template <bool LU_SMEM>
__device__ __forceinline__ FdpfLayout fdpf_layout(const DevPlan &P, const DevPlan *B, const BatchArgs &A,
                                                  unsigned char *dyn) {
    FdpfLayout L;
    double *x = reinterpret_cast<double *>(dyn);
    for (int k = 0; k < 2; ++k) {
        L.x[k] = x;
        L.lu[k] = LU_SMEM ? x + B[k].lu_offset : B[k].luval;
    }
    int *t = reinterpret_cast<int *>(dyn + fdpf_region_bytes(B[0], B[1], LU_SMEM));
    for (int k = 0; k < 2; ++k) {
        L.sbf[k] = t;
        t += B[k].fwd_nph + 1;
        L.sbb[k] = t;
        t += B[k].bwd_nph + 1;
        L.swf[k] = t;
        t += B[k].fwd_nph;
        L.swb[k] = t;
        t += B[k].bwd_nph;
    }
    unsigned char *slab = A.scratch + (size_t)blockIdx.x * (size_t)A.slab_bytes;
    L.V = reinterpret_cast<double2 *>(slab);
    L.T = L.V + P.n;
    L.Vm = reinterpret_cast<double *>(L.T + P.n);
    L.Va = L.Vm + P.n;
    return L;
}

// B x = b for one decoupled system: forward and backward programs over the constant factors,
// then the division by the pivots (the backward program keeps z undivided).
template <bool LU_SMEM>
__device__ __forceinline__ void fdpf_solve(const DevPlan &B, const FdpfLayout &L, int k, Trace &tr) {
    double *x = L.x[k];
    double *lu = const_cast<double *>(L.lu[k]);  // read only: substitutions do not write the LU
    run_lu_program<double, double, LU_SMEM>(B.fwd_cops, B.fwd_ops, L.sbf[k], L.swf[k], B.fwd_nph, B.m, lu, x, tr);
    run_lu_program<double, double, LU_SMEM>(B.bwd_cops, B.bwd_ops, L.sbb[k], L.swb[k], B.bwd_nph, B.m, lu, x, tr);
    for (int i = threadIdx.x; i < B.m; i += blockDim.x) x[i] = x[i] / lu[B.dpos[i]];
    __syncthreads();
}

// mis = (V conj(Ybus V) - Sbus + slack_absorbed w) / Vm: P into x at xP (which 0, for the next
// B' solve) or Q into x at xQ (which 1, for the next B'' solve); returns max(|P|, |Q|) and "some
// bus's mis is not finite" to every thread.
__device__ void fdpf_mismatch(const DevPlan &P, Shared &S, const double2 *__restrict__ V,
                              const double *__restrict__ Vm, const double2 *__restrict__ Sbus, double *x, int which,
                              double &norm, int &bad) {
    double lmax = 0.0;
    int lbad = 0;
    const double sa = S.slack_absorbed;
    for (int r = threadIdx.x; r < P.n; r += blockDim.x) {
        const double2 s = ybus_row_product(P, S, V, r);
        const double2 vr = V[r];
        const double2 sb = Sbus[r];
        double mr = vr.x * s.x + vr.y * s.y - sb.x;  // V * conj(I) - S + slack_absorbed * w
        double mi = vr.y * s.x - vr.x * s.y - sb.y;
        mr += sa * P.w[r];
        const double vm = Vm[r];
        mr /= vm;
        mi /= vm;
        lbad |= !isfinite(mr) || !isfinite(mi);
        const int ip = P.xP[r], iq = P.xQ[r];
        if (ip >= 0) {
            if (which == 0) x[ip] = mr;
            lmax = fmax(lmax, fabs(mr));
        }
        if (iq >= 0) {
            if (which == 1) x[iq] = mi;
            lmax = fmax(lmax, fabs(mi));
        }
    }
    block_norm(S, lmax, lbad, norm, bad);
}

// MAXT / MINB: launch bounds.  With the factors in global memory (read by every CTA of an SM
// through L1) small CTAs, many per SM, hide the latency of the substitution phases.
template <bool LU_SMEM, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) fdpf_batch_kernel(const DevPlan P0, const DevPlan B0, const DevPlan B1,
                                                                const BatchArgs A) {
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ Shared S;
    // the three plans in shared memory: indexed by system without copies of kernel parameters
    __shared__ __align__(16) DevPlan sp[3];
    const int tid = threadIdx.x;
    if (tid == 0) {
        sp[0] = P0;
        sp[1] = B0;
        sp[2] = B1;
    }
    __syncthreads();
    const DevPlan &P = sp[0];
    const DevPlan *B = sp + 1;
    const int n = P.n;
    const FdpfLayout L = fdpf_layout<LU_SMEM>(P, B, A, dyn);
    {
        for (int k = 0; k < 2; ++k) {
            const DevPlan &b = B[k];
            for (int i = tid; i <= b.fwd_nph; i += blockDim.x) L.sbf[k][i] = b.fwd_base[i];
            for (int i = tid; i <= b.bwd_nph; i += blockDim.x) L.sbb[k][i] = b.bwd_base[i];
            for (int i = tid; i < b.fwd_nph; i += blockDim.x) L.swf[k][i] = b.fwd_width[i];
            for (int i = tid; i < b.bwd_nph; i += blockDim.x) L.swb[k][i] = b.bwd_width[i];
            if (LU_SMEM)
                for (int i = tid; i < b.nnzLU; i += blockDim.x) L.x[k][b.lu_offset + i] = b.luval[i];
        }
    }
    __syncthreads();
    double2 *V = L.V, *T = L.T;
    double *Vm = L.Vm, *Va = L.Va;
    Trace tr{nullptr, 0, 0};
    for (;;) {
        if (tid == 0) S.job = atomicAdd(A.job_counter, 1);
        __syncthreads();
        const int job = S.job;
        __syncthreads();
        if (job >= A.njobs) break;
        const int first = A.job_first[job], count = A.job_count[job];
        for (int step = 0; step < count; ++step) {
            const int inst = first + step;
            const double2 *Sb = A.Sbus + (long long)inst * A.sbus_stride;
            if (step == 0 || !A.chain) {
                const double2 *v0 = A.V0 + (long long)inst * A.v0_stride;
                for (int b = tid; b < n; b += blockDim.x) V[b] = v0[b];
            }
            for (int b = tid; b < n; b += blockDim.x) {
                const double2 v = V[b];
                Vm[b] = cabs2(v);
                Va[b] = atan2(v.y, v.x);
            }
            if (tid == 0) {
                int k0 = 0, k1 = 0;
                if (A.ovr_ptr) {
                    k0 = A.ovr_ptr[inst];
                    k1 = A.ovr_ptr[inst + 1];
                }
                S.novr = k1 - k0 > kMaxOverrides ? -1 : k1 - k0;  // -1: too many to stage
            }
            __syncthreads();
            if (tid < S.novr) {
                const int k0 = A.ovr_ptr[inst];
                S.opos[tid] = A.ovr_pos[k0 + tid];
                S.oval[tid] = A.ovr_val[k0 + tid];
            }
            double ls = 0.0;
            for (int b = tid; b < n; b += blockDim.x) ls += Sb[b].x;
            const double tot = block_sum(S, ls);  // contains barriers
            if (tid == 0) S.slack_absorbed = tot;
            __syncthreads();
            if (S.novr < 0) {
                // more Ybus overrides than the kernel stages: not computed (start voltages out)
                double2 *vo = out_row(A, inst, n);
                for (int b = tid; b < n; b += blockDim.x) vo[b] = A.zero_failed ? make_double2(0.0, 0.0) : V[b];
                if (tid == 0) {
                    A.iters[inst] = 0;
                    A.errs[inst] = 8;  // NotInitError
                }
                __syncthreads();
                if (A.chain) {
                    for (int s2 = step + 1 + tid; s2 < count; s2 += blockDim.x) {
                        A.iters[first + s2] = 0;
                        A.errs[first + s2] = 8;
                    }
                    break;
                }
                continue;
            }
            double norm;
            int bad;
            fdpf_mismatch(P, S, V, Vm, Sb, L.x[0], 0, norm, bad);
            bool conv = !bad && norm < A.tol;
            int it = 0, err = 0;
            while (!conv && it < A.max_iter) {
                ++it;
                // P half-step
                fdpf_solve<LU_SMEM>(B[0], L, 0, tr);
                for (int b = tid; b < n; b += blockDim.x) {
                    double va = Va[b];
                    const int ia = P.xVa[b];
                    if (ia >= 0) va -= L.x[0][ia];
                    double sn, cs;
                    sincos(va, &sn, &cs);
                    T[b] = make_double2(cs, sn);
                    const double vm = Vm[b];
                    const double2 v = make_double2(vm * cs, vm * sn);
                    V[b] = v;
                    Vm[b] = cabs2(v);
                    Va[b] = atan2(v.y, v.x);
                }
                __syncthreads();
                fdpf_mismatch(P, S, V, Vm, Sb, L.x[0], 1, norm, bad);
                if (bad) {
                    err = 3;  // InifiniteValue
                    break;
                }
                if (norm < A.tol) {
                    conv = true;
                    break;
                }
                // Q half-step
                fdpf_solve<LU_SMEM>(B[1], L, 1, tr);
                for (int b = tid; b < n; b += blockDim.x) {
                    double vm = Vm[b];
                    const int im = P.xVm[b];
                    if (im >= 0) vm -= L.x[1][im];
                    const double2 t = T[b];
                    const double2 v = make_double2(vm * t.x, vm * t.y);
                    V[b] = v;
                    Vm[b] = cabs2(v);
                    Va[b] = atan2(v.y, v.x);
                }
                __syncthreads();
                fdpf_mismatch(P, S, V, Vm, Sb, L.x[0], 0, norm, bad);
                if (bad) {
                    // the reference notices the error after the next iteration's B' solve
                    err = 3;
                    if (it < A.max_iter) ++it;
                    break;
                }
                conv = norm < A.tol;
            }
            if (!conv && err == 0) err = 2;  // TooManyIterations
            double2 *vo = out_row(A, inst, n);
            const bool zero = A.zero_failed && err != 0;
            for (int b = tid; b < n; b += blockDim.x) vo[b] = zero ? make_double2(0.0, 0.0) : V[b];
            if (tid == 0) {
                A.iters[inst] = it;
                A.errs[inst] = err;
            }
            __syncthreads();
            if (A.chain && err != 0) {
                // the reference stops a time series at its first divergence
                for (int s2 = step + 1 + tid; s2 < count; s2 += blockDim.x) {
                    A.iters[first + s2] = 0;
                    A.errs[first + s2] = 8;  // NotInitError: not computed
                }
                break;
            }
        }
        __syncthreads();
    }
}

template <typename LT, typename XT, bool SM, bool RF, bool Q, int MAXT>
cudaError_t launch_variant_t(const DevPlan &P, const BatchArgs &A, const MultiArgs &M, int threads, int grid,
                             size_t smem, cudaStream_t st) {
    cudaError_t e = allow_max_smem(reinterpret_cast<const void *>(nr_batch_kernel<LT, XT, SM, RF, Q, MAXT>));
    if (e != cudaSuccess) return e;
    nr_batch_kernel<LT, XT, SM, RF, Q, MAXT><<<grid, threads, smem, st>>>(P, A, M);
    return cudaGetLastError();
}

// the variant of the smallest launch bound (512, 640, 768) that covers `threads`
template <typename LT, typename XT, bool SM, bool RF, bool Q>
cudaError_t launch_variant_q(const DevPlan &P, const BatchArgs &A, const MultiArgs &M, int threads, int grid,
                             size_t smem, cudaStream_t st) {
    if (threads > 768) return cudaErrorInvalidValue;
    if (threads > 640) return launch_variant_t<LT, XT, SM, RF, Q, 768>(P, A, M, threads, grid, smem, st);
    if (threads > 512) return launch_variant_t<LT, XT, SM, RF, Q, 640>(P, A, M, threads, grid, smem, st);
    return launch_variant_t<LT, XT, SM, RF, Q, 512>(P, A, M, threads, grid, smem, st);
}

template <typename LT, typename XT, bool SM, bool RF>
cudaError_t launch_variant(const DevPlan &P, const BatchArgs &A, const MultiArgs &M, int threads, int grid,
                           size_t smem, cudaStream_t st) {
    if (M.q.jobs != nullptr) return launch_variant_q<LT, XT, SM, RF, true>(P, A, M, threads, grid, smem, st);
    return launch_variant_q<LT, XT, SM, RF, false>(P, A, M, threads, grid, smem, st);
}

template <typename LT, typename XT, bool SM, bool RF>
int occupancy_variant(int threads, size_t smem) {
    int nb = 0;
    if (threads > 768) return 0;
    const void *fn = threads > 640   ? reinterpret_cast<const void *>(nr_batch_kernel<LT, XT, SM, RF, false, 768>)
                     : threads > 512 ? reinterpret_cast<const void *>(nr_batch_kernel<LT, XT, SM, RF, false, 640>)
                                     : reinterpret_cast<const void *>(nr_batch_kernel<LT, XT, SM, RF, false, 512>);
    if (allow_max_smem(fn) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess) return 0;
    return nb;
}

// Result rows in case order: row c = the converged voltages of compact instance map[c], or
// zeros (islanded case, map[c] < 0, or an instance that did not converge).
__global__ void scatter_case_rows(const double2 *__restrict__ src, const int *__restrict__ errs,
                                  const int *__restrict__ map, int ncases, int n, double2 *__restrict__ dst) {
    const long long total = (long long)ncases * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t / n), b = (int)(t - (long long)c * n);
        const int i = map[c];
        dst[t] = (i >= 0 && errs[i] == 0) ? src[(long long)i * n + b] : make_double2(0.0, 0.0);
    }
}

}  // namespace

cudaError_t launch_scatter_case_rows(const double2 *src, const int *errs, const int *map, int ncases, int n,
                                     double2 *dst, int num_sms, cudaStream_t st) {
    if (ncases <= 0) return cudaSuccess;
    scatter_case_rows<<<num_sms * 8, 256, 0, st>>>(src, errs, map, ncases, n, dst);
    return cudaGetLastError();
}

size_t slab_bytes(const DevPlan &P, int lu_bytes, bool lu_in_smem) {
    size_t bus = (((size_t)P.n * kBusSlabBytes + (size_t)P.m * 8) + 255) & ~(size_t)255;
    size_t lu = lu_in_smem ? 0 : (((size_t)P.nnzLU * lu_bytes + 255) & ~(size_t)255);
    // the dense tail block after the LU (global-memory LU plans only)
    size_t tail = lu_in_smem ? 0 : (((size_t)P.tail_k * (size_t)tail_ld(P.tail_k) * lu_bytes + 255) & ~(size_t)255);
    return bus + lu + tail;
}

size_t smem_bytes(const DevPlan &P, int lu_bytes, int x_bytes, bool lu_in_smem) {
    size_t xb = lu_in_smem ? (size_t)P.lu_offset * x_bytes : (((size_t)P.m * x_bytes + 15) & ~(size_t)15);
    size_t lb = lu_in_smem ? (((size_t)P.nnzLU * lu_bytes + 15) & ~(size_t)15) : 0;
    size_t bb = (size_t)(2 * (P.fac_nph + P.bwd_nph + P.fwd_nph) + 3) * sizeof(int);
    // staged operations of the narrow phases (make_layout places them after the tables)
    const size_t nb = P.nar_off[3] > 0 ? (((xb + lb + bb + 7) & ~(size_t)7) - (xb + lb + bb)) + (size_t)P.nar_off[3] * 8 : 0;
    // the dense tail's staging area, 16-byte aligned after the tables (global-memory LU)
    if (!lu_in_smem && P.tail_k > 0)
        return ((xb + lb + bb + nb + 7) & ~(size_t)7) + 16 + tail_smem_bytes(P.tail_k, lu_bytes);
    return xb + lb + bb + nb;
}

template <bool SM>
cudaError_t launch_dc_variant(const DevPlan &P, const BatchArgs &A, int threads, int grid, size_t smem,
                              cudaStream_t st) {
    cudaError_t e = allow_max_smem(reinterpret_cast<const void *>(dc_batch_kernel<SM>));
    if (e != cudaSuccess) return e;
    dc_batch_kernel<SM><<<grid, threads, smem, st>>>(P, A);
    return cudaGetLastError();
}

template <bool SM, int MAXT, int MINB>
cudaError_t launch_fdpf_variant(const DevPlan &P, const DevPlan &B0, const DevPlan &B1, const BatchArgs &A,
                                int threads, int grid, size_t smem, cudaStream_t st) {
    cudaError_t e = allow_max_smem(reinterpret_cast<const void *>(fdpf_batch_kernel<SM, MAXT, MINB>));
    if (e != cudaSuccess) return e;
    fdpf_batch_kernel<SM, MAXT, MINB><<<grid, threads, smem, st>>>(P, B0, B1, A);
    return cudaGetLastError();
}

// the kernel variant of a configuration: factors in shared memory (512 threads, 1 CTA per SM),
// or in global memory with 128-thread CTAs, 4 (registers unconstrained) or 8 (64 registers) per
// SM, or wider CTAs
const void *fdpf_kernel(bool lu_in_smem, int threads, int ctas_per_sm) {
    if (lu_in_smem) return reinterpret_cast<const void *>(fdpf_batch_kernel<true, 512, 1>);
    if (threads <= 128 && ctas_per_sm > 4) return reinterpret_cast<const void *>(fdpf_batch_kernel<false, 128, 8>);
    if (threads <= 128) return reinterpret_cast<const void *>(fdpf_batch_kernel<false, 128, 4>);
    return reinterpret_cast<const void *>(fdpf_batch_kernel<false, 512, 1>);
}

cudaError_t launch_fdpf_batch(const DevPlan &P, const DevPlan &B0, const DevPlan &B1, const BatchArgs &A,
                              int threads, int ctas_per_sm, int grid, size_t smem, cudaStream_t stream) {
    if (A.lu_in_smem) return launch_fdpf_variant<true, 512, 1>(P, B0, B1, A, threads, grid, smem, stream);
    if (threads <= 128 && ctas_per_sm > 4)
        return launch_fdpf_variant<false, 128, 8>(P, B0, B1, A, threads, grid, smem, stream);
    if (threads <= 128) return launch_fdpf_variant<false, 128, 4>(P, B0, B1, A, threads, grid, smem, stream);
    return launch_fdpf_variant<false, 512, 1>(P, B0, B1, A, threads, grid, smem, stream);
}

size_t fdpf_smem_bytes(const DevPlan &B0, const DevPlan &B1, bool lu_in_smem) {
    size_t b = fdpf_region_bytes(B0, B1, lu_in_smem);
    for (const DevPlan *B : {&B0, &B1}) b += (size_t)(2 * (B->fwd_nph + B->bwd_nph) + 2) * sizeof(int);
    return (b + 15) & ~(size_t)15;
}

size_t fdpf_slab_bytes(const DevPlan &P) { return ((size_t)P.n * 48 + 255) & ~(size_t)255; }

int fdpf_occupancy(bool lu_in_smem, int threads, int ctas_per_sm, size_t smem) {
    const void *fn = fdpf_kernel(lu_in_smem, threads, ctas_per_sm);
    int nb = 0;
    if (allow_max_smem(fn) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_nr_batch(const DevPlan &P, const BatchArgs &A, int precision, int threads, int grid,
                            size_t smem, cudaStream_t stream, const MultiArgs &M) {
    const bool sm = A.lu_in_smem != 0;
    if (P.dc) {
        if (M.segs != nullptr) return cudaErrorInvalidValue;  // DC plans run one plan per launch
        return sm ? launch_dc_variant<true>(P, A, threads, grid, smem, stream)
                  : launch_dc_variant<false>(P, A, threads, grid, smem, stream);
    }
    if (precision == 0) {
        return sm ? launch_variant<double, double, true, false>(P, A, M, threads, grid, smem, stream)
                  : launch_variant<double, double, false, false>(P, A, M, threads, grid, smem, stream);
    }
    if (A.refine)
        return sm ? launch_variant<float, float, true, true>(P, A, M, threads, grid, smem, stream)
                  : launch_variant<float, float, false, true>(P, A, M, threads, grid, smem, stream);
    return sm ? launch_variant<float, float, true, false>(P, A, M, threads, grid, smem, stream)
              : launch_variant<float, float, false, false>(P, A, M, threads, grid, smem, stream);
}

int nr_occupancy(int precision, bool lu_in_smem, bool refine, int threads, size_t smem) {
    if (precision == 0)
        return lu_in_smem ? occupancy_variant<double, double, true, false>(threads, smem)
                          : occupancy_variant<double, double, false, false>(threads, smem);
    if (refine)
        return lu_in_smem ? occupancy_variant<float, float, true, true>(threads, smem)
                          : occupancy_variant<float, float, false, true>(threads, smem);
    return lu_in_smem ? occupancy_variant<float, float, true, false>(threads, smem)
                      : occupancy_variant<float, float, false, false>(threads, smem);
}

}  // namespace l2g
